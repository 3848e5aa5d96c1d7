// Shared device helpers: vector types, stiffness constants, deterministic
// grid reductions and the device-resident control blocks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tpo.h"

namespace tpo {

constexpr unsigned FULL = 0xffffffffu;
constexpr int FIXED_X = 1;  // fixed-mask bits (one byte per node)
constexpr int FIXED_Y = 2;

// ---------------------------------------------------------------- constants
// Q4 element stiffness and the regularised inverse used by the element-block
// preconditioner, row-major 8x8, in both precisions. Indices are compile-time
// constants at every use, so each entry becomes a constant-bank operand.
__constant__ double c_ke[64];
__constant__ float c_ke_f[64];
__constant__ double c_kinv[64];
__constant__ float c_kinv_f[64];

// Square-Q4 structure of Ke: Ke = B0^T D B0 + ch (hx hx^T + hy hy^T), where B0
// is the strain matrix at the element centre and hx, hy the hourglass modes.
// {k11, k12, k33, ch, K00, K01} = {D11/4, D12/4, D33/4, ch, Ke[0][0], Ke[0][1]},
// derived from the uploaded Ke and checked against it entry by entry
// (tpo_set_stiffness). Every diagonal entry of such a Ke equals K00, and the
// x-y entry of corner a's 2x2 block is (-1)^a K01.
__constant__ double c_kst[6];
__constant__ float c_kst_f[6];
template <typename T> __device__ __forceinline__ T kst(int i);
template <> __device__ __forceinline__ double kst<double>(int i) { return c_kst[i]; }
template <> __device__ __forceinline__ float kst<float>(int i) { return c_kst_f[i]; }

template <typename T, bool INV> __device__ __forceinline__ T kmat(int i);
template <> __device__ __forceinline__ double kmat<double, false>(int i) { return c_ke[i]; }
template <> __device__ __forceinline__ float kmat<float, false>(int i) { return c_ke_f[i]; }
template <> __device__ __forceinline__ double kmat<double, true>(int i) { return c_kinv[i]; }
template <> __device__ __forceinline__ float kmat<float, true>(int i) { return c_kinv_f[i]; }

// ---------------------------------------------------------------- vectors
template <typename T> struct V2T;
template <> struct V2T<double> { typedef double2 type; };
template <> struct V2T<float> { typedef float2 type; };
template <typename T> using V2 = typename V2T<T>::type;

template <typename T> __device__ __forceinline__ V2<T> mk2(T x, T y) {
  V2<T> v;
  v.x = x;
  v.y = y;
  return v;
}
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }

template <typename T> __device__ __forceinline__ V2<T> ld2(const T *base, size_t node) {
  return reinterpret_cast<const V2<T> *>(base)[node];
}
template <typename T> __device__ __forceinline__ void st2(T *base, size_t node, V2<T> v) {
  reinterpret_cast<V2<T> *>(base)[node] = v;
}
template <typename T> __device__ __forceinline__ V2<T> shfl_up2(V2<T> v) {
  return mk2<T>(__shfl_up_sync(FULL, v.x, 1), __shfl_up_sync(FULL, v.y, 1));
}
template <typename T> __device__ __forceinline__ V2<T> shfl_down2(V2<T> v) {
  return mk2<T>(__shfl_down_sync(FULL, v.x, 1), __shfl_down_sync(FULL, v.y, 1));
}

// FP64 dot of two pairs (products of FP32 values are exact in FP64)
template <typename A, typename B>
__device__ __forceinline__ double dot2d(A a, B b) {
  return fma((double)a.x, (double)b.x, (double)a.y * (double)b.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// ---------------------------------------------------------------- control
// Device-resident PCG state. Fields are written only by the last CTA of a
// kernel (after every other CTA of that kernel has finished) and read by the
// CTAs of later kernels, so no CTA ever reads a field that is being written.
struct PcgCtl {
  double rz;        // r.z of the current residual
  double alpha;     // step length of the current iteration
  double beta;      // coefficient of the next direction update
  double rr;        // latest ||r||^2
  double pap;       // latest p.Ap
  double tol_sq;    // stop when rr < tol_sq
  double rupd2;     // mixed form: replace the residual when rr < rupd2 * rmax2 (0: plain)
  double rmax2;     // mixed form: ||r||^2 at the last FP64 residual evaluation
  int32_t it;       // completed updates
  int32_t status;   // TPO_SOLVE_* (or SOLVE_NEED_UPDATE)
  int32_t max_iter;
  int32_t first;    // 1: the next direction is p = z
  int32_t cont;     // mixed form: 1 after a residual replacement (keep p)
  int32_t err;      // nonzero: a bounded wait ran out (TMA pipeline)
  uint32_t counter; // last-CTA ticket
  int32_t since;    // mixed form: iterations since the last residual replacement
  int32_t phase;    // one-launch iteration: launches done (selects the ping-pong buffers)
};

// Outer refinement state of the mixed-precision solve.
struct OuterCtl {
  double rr;        // true FP64 ||f - K u||^2
  double tol_sq;
  int32_t it;       // residual evaluations so far
  int32_t status;   // TPO_SOLVE_*
  uint32_t counter;
  int32_t max_outer;  // residual evaluations allowed (then TPO_SOLVE_MAX_ITER)
};

struct OcCtl {
  double lo, hi, mid;
  double last_mid, change, vol;
  int32_t steps, done;
  uint32_t counter;
  int32_t pad;
};

struct SumCtl {
  uint32_t counter;
  int32_t pad;
};

// Block partials + last-CTA grid reduction, deterministic for a fixed grid:
// every CTA stores its NV partials (fixed in-block order), the CTA that
// finishes last re-reads all of them in block order and returns true with
// the grid totals in v[] (in every thread). Slot k is a max instead of a sum
// when bit k of MAXMASK is set. `part` holds NV*nblocks doubles. All threads
// of every CTA must call this (no early returns before it).
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *part, uint32_t *counter,
                                            int nb, int bid) {
  __shared__ double sm[NV * 32];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#define TPO_RED(k, a, b) (((MAXMASK >> (k)) & 1u) ? fmax((a), (b)) : (a) + (b))
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = ((MAXMASK >> k) & 1u) ? warp_max(v[k]) : warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sm[k * 32 + wid] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = sm[k * 32];
      for (int w = 1; w < nw; ++w) t = TPO_RED(k, t, sm[k * 32 + w]);
      part[(size_t)k * nb + bid] = t;
    }
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    s_last = (ticket == (unsigned)(nb - 1));
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;  // identity for sums; maxima here are of non-negative values
    for (int i = threadIdx.x; i < nb; i += blockDim.x) t = TPO_RED(k, t, __ldcg(part + (size_t)k * nb + i));
    v[k] = ((MAXMASK >> k) & 1u) ? warp_max(t) : warp_sum(t);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sm[k * 32 + wid] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = sm[k * 32];
    for (int w = 1; w < nw; ++w) t = TPO_RED(k, t, sm[k * 32 + w]);
    v[k] = t;
  }
#undef TPO_RED
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}
// over the whole launch grid
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *part, uint32_t *counter) {
  return grid_reduce<NV, MAXMASK>(v, part, counter, (int)(gridDim.x * gridDim.y),
                                  (int)(blockIdx.y * gridDim.x + blockIdx.x));
}

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

}  // namespace tpo
