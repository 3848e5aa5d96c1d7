// Design-side kernels of one OC iteration: the hat-weight filters, the
// compliance/sensitivity kernel and the device-side OC bisection.
#pragma once

#include "common.cuh"

namespace tpo {

// ---------------------------------------------------------------------------
// Hat-weight filter (reference optimizer/filter.py:22-171).
// The reference precomputes a neighbour list on the host; here each CTA
// derives the weights w(dx,dy) = rmin - sqrt(dx^2+dy^2) for the
// (2R+1)^2 box (R = ceil(rmin)) into shared memory, stages a 32x32 element
// tile plus an R-wide halo, and sums in the reference's neighbour order
// (dx outer, dy inner), skipping w <= 0 and out-of-domain neighbours.
// ---------------------------------------------------------------------------
constexpr int FT = 32;           // tile edge (elements)
constexpr int F_THREADS = 256;   // 32 rows x 8 columns of threads
constexpr int F_MAXR = 16;

enum FilterMode { F_DENSITY = 0, F_SENS = 1 };

// (bx, by) = (tile row, tile column) of this CTA
template <int MODE>
__device__ __forceinline__ void filter_run(int nx, int ny, double rmin, int R,
                                           const double *__restrict__ x,
                                           const double *__restrict__ rho,
                                           double *__restrict__ out, double *__restrict__ s_out,
                                           float *__restrict__ s32_out, double e_min, double pen,
                                           int bx, int by) {
  extern __shared__ double fsm[];
  const int W = 2 * R + 1;
  const int TW = FT + 2 * R;  // staged tile edge
  double *wt = fsm;           // W*W weights
  double *tile = fsm + W * W; // TW*TW values, index tx*TW + ty
  const int ex0 = by * FT, ey0 = bx * FT;

  for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
    const int dx = k / W - R, dy = k % W - R;
    wt[k] = rmin - sqrt((double)(dx * dx + dy * dy));
  }
  for (int k = threadIdx.x; k < TW * TW; k += blockDim.x) {
    const int tx = k / TW, ty = k % TW;
    const int gx = ex0 - R + tx, gy = ey0 - R + ty;
    double v = 0.0;
    if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
      const size_t e = (size_t)gx * ny + gy;
      v = (MODE == F_SENS) ? rho[e] * x[e] : x[e];
    }
    tile[k] = v;
  }
  __syncthreads();

  const int ty = threadIdx.x & 31;
  const int ey = ey0 + ty;
  for (int tx = threadIdx.x >> 5; tx < FT; tx += F_THREADS / 32) {
    const int ex = ex0 + tx;
    if (ex >= nx || ey >= ny) continue;
    double num = 0.0, den = 0.0;
    for (int dx = -R; dx <= R; ++dx) {
      const int jx = ex + dx;
      if (jx < 0 || jx >= nx) continue;
      const double *trow = tile + (size_t)(tx + R + dx) * TW + (ty + R);
      const double *wrow = wt + (dx + R) * W + R;
      for (int dy = -R; dy <= R; ++dy) {
        const double w = wrow[dy];
        const int jy = ey + dy;
        if (w > 0.0 && jy >= 0 && jy < ny) {
          num = fma(w, trow[dy], num);
          den += w;
        }
      }
    }
    const size_t e = (size_t)ex * ny + ey;
    double o;
    if (MODE == F_SENS) {
      o = num / (rho[e] * den + 1e-20);
    } else {
      o = num / (den + 1e-20);
      if (s_out || s32_out) {
        const double s = e_min + pow(o, pen) * (1.0 - e_min);
        if (s_out) s_out[e] = s;
        if (s32_out) s32_out[e] = (float)s;
      }
    }
    out[e] = o;
  }
}
template <int MODE>
__global__ void __launch_bounds__(F_THREADS)
    k_filter(int nx, int ny, double rmin, int R, const double *__restrict__ x,
             const double *__restrict__ rho, double *__restrict__ out,
             double *__restrict__ s_out, float *__restrict__ s32_out, double e_min,
             double pen) {
  filter_run<MODE>(nx, ny, rmin, R, x, rho, out, s_out, s32_out, e_min, pen, blockIdx.x,
                   blockIdx.y);
}

// ---------------------------------------------------------------------------
// Compliance and sensitivity (reference fem/kernels.py:234-272):
//   uKu_e = u_e^T Ke u_e, dc_e = -p rho_e^(p-1) (1 - e_min) uKu_e,
//   c = sum_e (e_min + rho_e^p (1 - e_min)) uKu_e.
// Lane = element row; each thread walks a strip of SL element columns.
// ---------------------------------------------------------------------------
constexpr int S_THREADS = 128;
constexpr int SL = 16;

__device__ __forceinline__ void sensitivity_run(int nx, int ny, double e_min, double pen,
                                                const double *__restrict__ rho,
                                                const double *__restrict__ u,
                                                double *__restrict__ dc, double *part, SumCtl *ctl,
                                                double *c_out, int bx, int by, int nb, int bid) {
  const int ey = bx * blockDim.x + threadIdx.x;
  const int x0 = by * SL;
  const int x1 = min(x0 + SL, nx);
  const size_t ny1 = (size_t)ny + 1;
  double acc[1] = {0.0};
  if (ey < ny) {
    double2 lo = reinterpret_cast<const double2 *>(u)[(size_t)x0 * ny1 + ey];
    double2 hi = reinterpret_cast<const double2 *>(u)[(size_t)x0 * ny1 + ey + 1];
    for (int ex = x0; ex < x1; ++ex) {
      const double2 rlo = reinterpret_cast<const double2 *>(u)[(size_t)(ex + 1) * ny1 + ey];
      const double2 rhi = reinterpret_cast<const double2 *>(u)[(size_t)(ex + 1) * ny1 + ey + 1];
      const double ue[8] = {lo.x, lo.y, rlo.x, rlo.y, rhi.x, rhi.y, hi.x, hi.y};
      double uku = 0.0;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        double ku = c_ke[i * 8] * ue[0];
#pragma unroll
        for (int j = 1; j < 8; ++j) ku = fma(c_ke[i * 8 + j], ue[j], ku);
        uku = fma(ue[i], ku, uku);
      }
      const size_t e = (size_t)ex * ny + ey;
      const double r = rho[e];
      dc[e] = -pen * pow(r, pen - 1.0) * (1.0 - e_min) * uku;
      acc[0] += (e_min + pow(r, pen) * (1.0 - e_min)) * uku;
      lo = rlo;
      hi = rhi;
    }
  }
  if (!grid_reduce<1>(acc, part, &ctl->counter, nb, bid)) return;
  if (threadIdx.x == 0) *c_out = acc[0];
}
__global__ void __launch_bounds__(S_THREADS)
    k_sensitivity(int nx, int ny, double e_min, double pen, const double *__restrict__ rho,
                  const double *__restrict__ u, double *__restrict__ dc, double *part,
                  SumCtl *ctl, double *c_out) {
  sensitivity_run(nx, ny, e_min, pen, rho, u, dc, part, ctl, c_out, blockIdx.x, blockIdx.y,
                  gridDim.x * gridDim.y, blockIdx.y * gridDim.x + blockIdx.x);
}

// ---------------------------------------------------------------------------
// OC update (reference optimizer/oc.py:21-93). One launch per bisection step;
// the step's last CTA reduces the volume, moves lo/hi and decides whether to
// stop, so lambda never visits the host. k_oc_final writes the density of the
// last midpoint evaluated.
// ---------------------------------------------------------------------------
constexpr int OC_THREADS = 256;
constexpr int OC_MAX_STEPS = 50;

__device__ __forceinline__ double oc_candidate(double r, double d, double dvv, double lam,
                                               double move) {
  const double be = fmax(-d / (lam * dvv + 1e-20), 0.0);
  const double cand = r * sqrt(be);
  const double lo = fmax(0.001, r - move);
  const double hi = fmin(1.0, r + move);
  return fmax(lo, fmin(hi, cand));
}

__device__ __forceinline__ void oc_init_run(OcCtl *ctl) {
  ctl->lo = 0.0;
  ctl->hi = 1e9;
  ctl->mid = 0.5 * (0.0 + 1e9);
  ctl->last_mid = 0.0;
  ctl->change = 0.0;
  ctl->vol = 0.0;
  ctl->steps = 0;
  ctl->done = 0;
  ctl->counter = 0u;
}
__global__ void k_oc_init(OcCtl *ctl) { oc_init_run(ctl); }

__device__ __forceinline__ void oc_step_run(int n, double volfrac, double move,
                                            const double *__restrict__ rho,
                                            const double *__restrict__ dc,
                                            const double *__restrict__ dv, double *part,
                                            OcCtl *ctl, int bx, int gx) {
  if (ctl->done) return;
  const double lam = ctl->mid;
  double acc[2] = {0.0, 0.0};  // sum of new densities, max |change|
  for (int e = bx * blockDim.x + threadIdx.x; e < n; e += gx * blockDim.x) {
    const double r = rho[e];
    const double nw = oc_candidate(r, dc[e], dv ? dv[e] : 1.0, lam, move);
    acc[0] += nw;
    acc[1] = fmax(acc[1], fabs(nw - r));
  }
  if (!grid_reduce<2, 2u>(acc, part, &ctl->counter, gx, bx)) return;
  if (threadIdx.x != 0) return;
  const double chg = acc[1];
  const double vol = acc[0] / n;
  ctl->last_mid = lam;
  ctl->change = chg;
  ctl->vol = vol;
  ctl->steps += 1;
  if (vol > volfrac) ctl->lo = lam; else ctl->hi = lam;
  if ((ctl->hi - ctl->lo) / (ctl->hi + ctl->lo + 1e-30) < 1e-4 || ctl->steps >= OC_MAX_STEPS) {
    ctl->done = 1;
  } else {
    ctl->mid = 0.5 * (ctl->lo + ctl->hi);
  }
}

__global__ void __launch_bounds__(OC_THREADS)
    k_oc_step(int n, double volfrac, double move, const double *__restrict__ rho,
              const double *__restrict__ dc, const double *__restrict__ dv, double *part,
              OcCtl *ctl) {
  oc_step_run(n, volfrac, move, rho, dc, dv, part, ctl, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ void oc_final_run(int n, double move, const double *rho_in,
                                             const double *__restrict__ dc,
                                             const double *__restrict__ dv, double *rho_out,
                                             const OcCtl *ctl, double *result, int bx, int gx) {
  const double lam = ctl->last_mid;
  for (int e = bx * blockDim.x + threadIdx.x; e < n; e += gx * blockDim.x) {
    const double r = rho_in[e];
    rho_out[e] = oc_candidate(r, dc[e], dv ? dv[e] : 1.0, lam, move);
  }
  if (bx == 0 && threadIdx.x == 0 && result) {
    result[0] = ctl->change;
    result[1] = ctl->vol;
    result[2] = ctl->last_mid;
    result[3] = (double)ctl->steps;
  }
}
__global__ void k_oc_final(int n, double move, const double *rho_in, const double *__restrict__ dc,
                           const double *__restrict__ dv, double *rho_out, const OcCtl *ctl,
                           double *result) {
  oc_final_run(n, move, rho_in, dc, dv, rho_out, ctl, result, blockIdx.x, gridDim.x);
}

}  // namespace tpo
