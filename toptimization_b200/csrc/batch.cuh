// Batched designs: one launch per kernel step covers every design of a batch.
//
// Each design occupies a slot with a device record (BDesign) holding its
// sizes, parameters, its resident state (design and physical density,
// sensitivities, displacement, the padded PCG vectors of the mixed form, the
// control blocks of the PCG, the OC bisection and the compliance sum) and its
// OC-iteration history. A batched kernel is launched with a 1-D grid; every
// kernel kind has a job table that maps a contiguous range of CTAs to one
// design and gives that design's local launch geometry (gx x gy CTAs). A CTA
// finds its job by binary search over the range starts, derives its local
// block (bx, by) and runs the same device code as the single-design kernel
// (tstencil_run, update_run, filter_run, ...). Reductions are per design: each
// design has its own partial-sum buffer and ticket counter, and its last CTA
// finishes its step.
//
// A design's launch geometry depends only on its own size and on the batch's
// tile parameters, never on the other designs in the batch, so a design's
// arithmetic (and its reduction order) is the same alone and in any mix.
//
// One OC iteration of a design (reference optimizer/simp.py:141-219) runs in
// three phases. PRE: density filter -> SIMP scales -> control init. SOLVE:
// PCG of the mixed form (FP64 residual replacement, then steps of direction
// + update) until its solve stops. POST: displacement unpack -> sensitivity
// and compliance -> dc filter -> OC bisection and update -> bookkeeping
// (history row, iteration count, stop rule), back to PRE. Every batched
// kernel acts only on the designs in its phase, so designs at different
// stages share the same launches (continuous batching), and a design's own
// sequence of operations is the same whatever the others are doing.
#pragma once

#include "common.cuh"
#include "design.cuh"
#include "layout.cuh"
#include "pcg.cuh"

namespace tpo {

// device record of one design slot
// phases of a design within its current OC iteration
enum BPhase { PH_PRE = 0, PH_SOLVE = 1, PH_POST = 2 };

struct BDesign {
  int nx, ny, P, active;       // active: OC iterations remain
  int it, max_it, R, max_cg;   // OC iterations done / requested, filter radius, PCG cap
  int max_outer, phase;        // phase: BPhase
  int period;                  // takes the PCG steps i of a loop body with i % period == 0 (0, 1: all)
  int pad1;
  double e_min, pen, volfrac, move, rmin, tol;  // tol: early stop on change (0: none)
  double tol_sq, rupd2;        // PCG stop (true residual) and replacement thresholds
  // compact fields, reference numbering
  double *rho, *rho_phys, *dc, *dc_filt, *u;
  double *hist;                // max_it rows of kBatchHist values
  // padded PCG state of the mixed form
  uint8_t *mask;
  double *up, *fp, *s64;
  float *s32, *fr, *fpa, *fpb, *fap, *fz;  // fz = M r, written by the update kernel
  PcgCtl *ctl;
  OuterCtl *octl;
  double *part;
  // compliance sum
  SumCtl *sc;
  double *spart;
  double *scal;                // [0] compliance, [1..4] OC result (change, volume, lambda, steps)
};

// history row per OC iteration: compliance, volume, change, PCG iterations,
// FP64 residual evaluations, PCG status
constexpr int kBatchHist = 6;

struct BJob {
  int cta0;    // first CTA of this design in the launch
  int gx, gy;  // local grid
  int slot;
  int L;       // strip length (stencil / update kinds)
  int pad;
};

__device__ __forceinline__ const BJob &find_job(const BJob *__restrict__ jobs, int n) {
  int lo = 0, hi = n - 1;
  const int b = (int)blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].cta0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return jobs[lo];
}

// ---------------------------------------------------------------- kernels
// density filter (which = 0: rho -> rho_phys) or dc filter (which = 1: dc -> dc_filt)
__global__ void __launch_bounds__(F_THREADS)
    kb_filter(const BJob *jobs, int nj, const BDesign *ds, int which) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || D.phase != (which ? PH_POST : PH_PRE)) return;
  const int loc = blockIdx.x - J.cta0;
  const double *x = which ? D.dc : D.rho;
  double *out = which ? D.dc_filt : D.rho_phys;
  filter_run<F_DENSITY>(D.nx, D.ny, D.rmin, D.R, x, nullptr, out, nullptr, nullptr, 0.0, 0.0,
                        loc % J.gx, loc / J.gx);
}

__global__ void kb_scales(const BJob *jobs, int nj, const BDesign *ds) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || D.phase != PH_PRE) return;
  scales_run(D.nx, D.ny, D.P, D.rho_phys, D.e_min, D.pen, 0.0, D.s64, D.s32, nullptr, nullptr,
             blockIdx.x - J.cta0, J.gx);
}

// one thread per slot: PCG control blocks of a new OC iteration; PRE -> SOLVE
__global__ void kb_init(BDesign *ds, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BDesign &D = ds[i];
  if (!D.active || D.phase != PH_PRE) return;
  ctl_init_run(D.ctl, D.tol_sq, D.rupd2, D.max_cg, D.octl, D.tol_sq, D.max_outer);
  D.phase = PH_SOLVE;
}

// one thread per slot: SOLVE -> POST once the design's solve has stopped
__global__ void kb_mark(BDesign *ds, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BDesign &D = ds[i];
  if (!D.active || D.phase != PH_SOLVE) return;
  const int st = D.ctl->status;
  if (st != TPO_SOLVE_RUNNING && st != SOLVE_NEED_UPDATE) D.phase = PH_POST;
}

// stencil ring of the batched kernels: kBatchNG slots of kBatchG columns
constexpr int kBatchG = 2, kBatchNG = 4;

template <int PRE>
__global__ void __launch_bounds__(TS_THREADS) kb_resx(const BJob *jobs, int nj, const BDesign *ds) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active) return;
  TsArgs a{};
  a.nx = D.nx;
  a.ny = D.ny;
  a.P = D.P;
  a.s = D.s64;
  a.mask = D.mask;
  a.a = D.up;
  a.uw = D.up;
  a.f = D.fp;
  a.out = D.fr;
  a.part = D.part;
  a.ctl = D.ctl;
  a.octl = D.octl;
  a.err = &D.ctl->err;
  const int loc = blockIdx.x - J.cta0;
  tstencil_run<double, double, M_RESX, PRE, kBatchG, kBatchNG>(a, J.L, loc % J.gx, loc / J.gx, J.gx * J.gy,
                                                  loc);
}

template <int PRE>
__global__ void __launch_bounds__(TS_THREADS) kb_dir(const BJob *jobs, int nj, const BDesign *ds,
                                                     int step) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || (D.period > 1 && step % D.period != 0)) return;
  TsArgs a{};
  a.nx = D.nx;
  a.ny = D.ny;
  a.P = D.P;
  a.s = D.s32;
  a.mask = D.mask;
  a.a = D.fz;  // z = M r from the update kernel (or the pass after a replacement)
  a.pa = D.fpa;
  a.pb = D.fpb;
  a.out = D.fap;
  a.part = D.part;
  a.ctl = D.ctl;
  a.err = &D.ctl->err;
  const int loc = blockIdx.x - J.cta0;
  tstencil_run<float, double, M_DIR, TPO_PRECOND_BLOCK_JACOBI, kBatchG, kBatchNG>(
      a, J.L, loc % J.gx, loc / J.gx, J.gx * J.gy, loc);
}

// z = M r for every design in its solve (after the FP64 residual replacement
// of a loop body; for the others it rewrites the z their update stored)
template <int PRE>
__global__ void __launch_bounds__(UF_THREADS) kb_pre(const BJob *jobs, int nj, const BDesign *ds) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || D.phase != PH_SOLVE || D.ctl->status != TPO_SOLVE_RUNNING) return;
  precond_flat_run<float, double, PRE>(D.nx, D.ny, D.P, D.s32, D.mask, D.fr, D.fz,
                                       blockIdx.x - J.cta0, J.gx);
}

template <int PRE>
__global__ void __launch_bounds__(UF_THREADS) kb_update(const BJob *jobs, int nj,
                                                        const BDesign *ds, int step) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || (D.period > 1 && step % D.period != 0)) return;
  UpdArgs a{};
  a.nx = D.nx;
  a.ny = D.ny;
  a.P = D.P;
  a.s = D.s32;
  a.mask = D.mask;
  a.u = D.up;
  a.r = D.fr;
  a.ap = D.fap;
  a.pa = D.fpa;
  a.pb = D.fpb;
  a.part = D.part;
  a.ctl = D.ctl;
  a.z = D.fz;
  const int loc = blockIdx.x - J.cta0;
  update_flat_run<float, double, PRE, double>(a, loc, J.gx, J.gx, loc);
}

// Is any solve of the batch still going? flag[0] = 1 if so; flag[1] = 1 when
// the body limit stopped a loop that still had work (an error). Inside a CUDA
// graph it also sets the while-node condition.
__global__ void kb_cond(const BDesign *ds, int n, int *flag, unsigned *bodies,
                        unsigned max_bodies, cudaGraphConditionalHandle h, int use_h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const BDesign &D = ds[i];
    if (!D.active || D.phase != PH_SOLVE) continue;
    const int st = D.ctl->status;
    if ((st == TPO_SOLVE_RUNNING || st == SOLVE_NEED_UPDATE) && D.ctl->err == 0) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned b = *bodies + 1u;
    *bodies = b;
    const int go = any && b < max_bodies;
    if (any && !go) flag[1] = 1;
    flag[0] = go;
    if (use_h) cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

__global__ void kb_unpack(const BJob *jobs, int nj, const BDesign *ds) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || D.phase != PH_POST) return;
  unpack_nodes_run(D.nx, D.ny, D.P, D.up, D.u, blockIdx.x - J.cta0, J.gx);
}

__global__ void __launch_bounds__(S_THREADS) kb_sens(const BJob *jobs, int nj, const BDesign *ds) {
  const BJob &J = find_job(jobs, nj);
  const BDesign &D = ds[J.slot];
  if (!D.active || D.phase != PH_POST) return;
  const int loc = blockIdx.x - J.cta0;
  sensitivity_run(D.nx, D.ny, D.e_min, D.pen, D.rho_phys, D.u, D.dc, D.spart, D.sc, D.scal,
                  loc % J.gx, loc / J.gx, J.gx * J.gy, loc);
}

// OC update of one design per CTA (reference optimizer/oc.py:21-93, same
// rules as k_oc_step / k_oc_final): bisection on lambda in [0, 1e9], at most
// OC_MAX_STEPS midpoints, stop when (hi - lo) / (hi + lo) < 1e-4; the density
// is updated in place with the last midpoint evaluated. One CTA loops over the
// steps, so the whole bisection is one launch for every design of the batch.
constexpr int OCB_THREADS = 1024;
__global__ void __launch_bounds__(OCB_THREADS) kb_oc(BDesign *ds, int n) {
  if ((int)blockIdx.x >= n) return;
  BDesign &D = ds[blockIdx.x];
  if (!D.active || D.phase != PH_POST) return;
  __shared__ double red[2][OCB_THREADS / 32];
  __shared__ double res[2];
  const int ne = D.nx * D.ny;
  const double *rho = D.rho;  // updated in place at the end
  const double *__restrict__ dcf = D.dc_filt;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double lo = 0.0, hi = 1e9, lam = 0.5 * (0.0 + 1e9), last = 0.0, chg = 0.0, vol = 0.0;
  int steps = 0;
  for (;;) {
    double sum = 0.0, mx = 0.0;
    for (int e = threadIdx.x; e < ne; e += OCB_THREADS) {
      const double r = rho[e];
      const double nw = oc_candidate(r, dcf[e], 1.0, lam, D.move);
      sum += nw;
      mx = fmax(mx, fabs(nw - r));
    }
    sum = warp_sum(sum);
    mx = warp_max(mx);
    if (lane == 0) {
      red[0][wid] = sum;
      red[1][wid] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = red[0][0], m = red[1][0];
      for (int w = 1; w < OCB_THREADS / 32; ++w) {
        t += red[0][w];
        m = fmax(m, red[1][w]);
      }
      res[0] = t;
      res[1] = m;
    }
    __syncthreads();
    last = lam;
    chg = res[1];
    vol = res[0] / ne;
    steps += 1;
    if (vol > D.volfrac) lo = lam; else hi = lam;
    if ((hi - lo) / (hi + lo + 1e-30) < 1e-4 || steps >= OC_MAX_STEPS) break;
    lam = 0.5 * (lo + hi);
    __syncthreads();  // res[] is rewritten by the next step
  }
  for (int e = threadIdx.x; e < ne; e += OCB_THREADS)
    D.rho[e] = oc_candidate(rho[e], dcf[e], 1.0, last, D.move);
  if (threadIdx.x == 0) {
    D.scal[1] = chg;
    D.scal[2] = vol;
    D.scal[3] = last;
    D.scal[4] = (double)steps;
  }
}

// one thread per slot: history row, iteration count, stop rule
// (reference optimizer/simp.py:216-219: stop when it > 5 and change < tol);
// status[2i..2i+1] = (it, active) for the host, *err |= 1 on a pipeline timeout
__global__ void kb_finish(BDesign *ds, int n, int *status, int *err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BDesign &D = ds[i];
  if (!D.active || D.phase != PH_POST) return;
  if (D.ctl->err) atomicOr(err, 1);
  double *h = D.hist + (size_t)D.it * kBatchHist;
  h[0] = D.scal[0];
  h[1] = D.scal[2];
  h[2] = D.scal[1];
  h[3] = (double)D.ctl->it;
  h[4] = (double)D.octl->it;
  h[5] = (double)D.ctl->status;
  D.it += 1;
  D.phase = PH_PRE;
  if (D.it >= D.max_it || (D.tol > 0.0 && D.it > 5 && D.scal[1] < D.tol)) D.active = 0;
  status[2 * i] = D.it;
  status[2 * i + 1] = D.active;
}

}  // namespace tpo
