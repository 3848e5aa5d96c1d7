// PCG kernels on the padded layout (layout.cuh) for the two-launch forms
// (the mixed form, the element-block preconditioner, and the reference's own
// recurrence; the one-launch FP64 iteration is in cgstep.cuh):
//   k_tstencil<DIR>  p = z + beta p (z stored by the update kernel or by the
//                    element-block preconditioner), Ap = K p, p.Ap;
//                    its last CTA sets alpha (or flags a breakdown).
//   k_update_flat / k_blockpre<UPDATE>
//                    u += alpha p, r -= alpha Ap, z = M r (stored), r.z,
//                    ||r||^2; its last CTA decides convergence / refinement
//                    and beta.
// alpha, beta and the stop test never leave the device (PcgCtl). Every CTA
// reads the status word first and returns at once when the solve is over, so
// a host may enqueue more iterations than needed.
//
// T is the storage type of the Krylov vectors (r, p, Ap, z) and scales, C the
// arithmetic type, X the type of the solution u: <double,double,double> for
// the plain FP64 solve, <float,double,double> for the mixed form (FP32 bytes
// for the Krylov vectors, FP64 arithmetic, dot products and solution). u stays
// FP64 in the mixed form: accumulating it in FP32 between residual
// replacements injects rounding noise of relative size 2^-24 into every
// replaced residual, which the iteration then has to remove again.
//
// k_tstencil: each CTA owns 120 grid rows (4 warps x 30; a warp's first and
// last lane are halo rows) and walks a strip of L node columns. Column windows
// of every input are staged into shared memory by TMA bulk copies
// (cp.async.bulk) in groups of G columns, NG groups in flight, completion on
// one mbarrier per ring slot; a fifth warp produces, four warps consume. Each
// thread keeps the 3x3 neighbourhood of transformed nodal values in registers,
// y neighbours arrive by warp shuffles. Strips overlap by two columns; values
// there are recomputed from the inputs, never read from another strip's
// output, and the direction p ping-pongs between two buffers so no CTA
// overwrites what another still reads.
#pragma once

#include "common.cuh"
#include "layout.cuh"
#include "stencil.cuh"

namespace tpo {

constexpr int ST_THREADS = WPC * 32;  // 128 (k_blockpre)
constexpr int TS_THREADS = ST_THREADS + 32;  // stencil: 4 consumer warps + 1 producer warp

enum StMode { M_RAW = 0, M_DIR = 1, M_RES = 2, M_RESX = 3 };

// solve status used only between the inner kernels and the host of the mixed
// form: the FP32 residual dropped enough, an FP64 residual replacement is due
constexpr int SOLVE_NEED_UPDATE = 6;
constexpr int kReplaceEvery = 1000;  // mixed form: longest run between FP64 residuals
constexpr int ERR_TMA_TIMEOUT = 1;

template <typename C, typename T> __device__ __forceinline__ V2<C> cvt2(V2<T> v) {
  return mk2<C>(C(v.x), C(v.y));
}

struct TsArgs {
  int nx, ny, P;
  const void *s;          // element scales (T, padded)
  const uint8_t *mask;    // fixed mask (padded)
  const void *a;          // RAW: x; DIR: r (point precond) or z (block); RES/RESX: u
  void *pa, *pb;          // DIR: direction ping-pong (T)
  void *out;              // RAW: y; DIR: Ap; RES: r; RESX: inner r (float)
  void *uw;               // RES/RESX: u written back with fixed DOFs zeroed
  const void *f;          // RES/RESX: right-hand side (T)
  double *part;
  PcgCtl *ctl;
  OuterCtl *octl;
  double *result;         // RAW: optional p.Ap
  int *err;               // TMA timeout flag
  void *out2;             // RESX: if set, the residual buffer of odd iterations (out: even)
  int withhold1;          // failure tests only: g + 1 withholds the copies of column group g
};

template <typename T, int MODE> struct TsGeom {
  static constexpr bool HAS_B = MODE == M_DIR;
  static constexpr int CNB = N_WIN * 2 * (int)sizeof(T);   // node bytes per column
  static constexpr int CEB = EWin<T>::N * (int)sizeof(T);  // element bytes per column
  static constexpr int CMB = M_WIN;                        // mask bytes per column
  template <int G> __host__ __device__ static constexpr int slot_bytes() {
    return G * (CNB * (HAS_B ? 2 : 1) + CEB + CMB);
  }
};

// (bx, by) = (row block, strip) of this CTA, nb / bid = CTAs of the solve and
// this CTA's index among them (a batched launch runs many solves at once)
template <typename T, typename C, int MODE, int PRE, int G, int NG>
__device__ __forceinline__ void tstencil_run(const TsArgs &a, int L, int bx, int by, int nb,
                                             int bid) {
  using Geo = TsGeom<T, MODE>;
  constexpr int NV = (MODE == M_RAW || MODE == M_DIR) ? 1 : (MODE == M_RES ? 2 : 3);
  constexpr int SLOT = Geo::template slot_bytes<G>();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[NG];   // group staged (TMA transaction bytes)
  __shared__ __align__(8) uint64_t empty[NG];  // group consumed by all warps

  PcgCtl *ctl = a.ctl;
  C beta = C(0);
  bool first = true;
  int parity = 0;
  if constexpr (MODE == M_DIR) {
    if (ctl->status != TPO_SOLVE_RUNNING) return;
    beta = C(ctl->beta);
    first = ctl->first != 0;
    parity = ctl->it & 1;
  }
  if constexpr (MODE == M_RESX) {
    // runs only when the inner iteration asked for a residual replacement
    // (or before the first iteration): a batched launch reaches every solve
    if (ctl->status != SOLVE_NEED_UPDATE || a.octl->status != TPO_SOLVE_RUNNING) return;
  }
  const int nx = a.nx, ny = a.ny, P = a.P;
  const int Y0 = bx * RPC;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int y = Y0 + wid * RPW - 1 + lane;
  const bool own_row = lane >= 1 && lane <= RPW && y <= ny;
  const int x0 = by * L;
  const int x1 = min(x0 + L, nx + 1);
  // Only a direction kernel that rebuilds a point preconditioner at node
  // x0-1 needs element column x0-2: it stages that column's scales alone.
  // Every other mode starts at x0-1 with nodes and scales.
  constexpr bool SCALE_COL = MODE == M_DIR && PRE != TPO_PRECOND_BLOCK_JACOBI;
  const int cA = x0 - (SCALE_COL ? 2 : 1);  // first staged column
  const int NC = x1 - cA + 1;               // staged columns cA..x1
  const int NGRP = (NC + G - 1) / G;
  const int ms = (Y0 + LEAD - 1) & ~15;  // first staged mask byte of a column

  const T *gs = static_cast<const T *>(a.s);
  const T *ga = static_cast<const T *>(a.a);
  T *src_p = nullptr, *dst_p = nullptr;
  if constexpr (MODE == M_DIR) {
    src_p = static_cast<T *>(parity ? a.pb : a.pa);
    dst_p = static_cast<T *>(parity ? a.pa : a.pb);
  }

  // ---- producer (thread 0): stage group g into ring slot g % NG. A slot is
  // reused only after every warp has released the group it held (empty[]),
  // and the producer refills with a lag of one group, so warps may drift
  // apart by a group without waiting for each other.
  auto issue = [&](int g) {
    if (g + 1 == a.withhold1) return;  // failure tests: the group's wait must run out
    unsigned char *sb = smem + (g % NG) * SLOT;
    unsigned bytes = 0;
    for (int k = 0; k < G; ++k) {
      const int c = cA + g * G + k;
      if (c > x1) break;
      if ((!SCALE_COL || c > cA) && c >= 0 && c <= nx)
        bytes += Geo::CNB * (Geo::HAS_B ? 2 : 1) + Geo::CMB;
      if (c >= 0 && c < nx) bytes += Geo::CEB;
    }
    mbar_arrive_expect_tx(&full[g % NG], bytes);
    for (int k = 0; k < G; ++k) {
      const int c = cA + g * G + k;
      if (c > x1) break;
      if ((!SCALE_COL || c > cA) && c >= 0 && c <= nx) {
        const size_t col = (size_t)c * P + Y0 + N_OFF;
        bulk_g2s(sb + k * Geo::CNB, ga + 2 * col, Geo::CNB, &full[g % NG]);
        if constexpr (Geo::HAS_B)
          bulk_g2s(sb + G * Geo::CNB + k * Geo::CNB, src_p + 2 * col, Geo::CNB, &full[g % NG]);
        bulk_g2s(sb + G * Geo::CNB * (Geo::HAS_B ? 2 : 1) + G * Geo::CEB + k * Geo::CMB,
                 a.mask + (size_t)c * P + ms, Geo::CMB, &full[g % NG]);
      }
      if (c >= 0 && c < nx) {
        bulk_g2s(sb + G * Geo::CNB * (Geo::HAS_B ? 2 : 1) + k * Geo::CEB,
                 gs + (size_t)c * P + Y0 + EWin<T>::OFF, Geo::CEB, &full[g % NG]);
      }
    }
  };
  bool ok = true;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NG; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], WPC);
    }
    fence_mbar_init();
  }
  __syncthreads();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;

  if (wid == WPC) {
    // ---- producer warp: refill slot g % NG with group g once its previous
    // tenant (g - NG) has been released by every consumer warp
    if (lane == 0) {
      int issued = 0;
      for (int g = 0; g < NGRP; ++g) {
        if (g >= NG)
          ok = mbar_wait_bounded(&empty[g % NG], ((g / NG) - 1) & 1, a.err, ERR_TMA_TIMEOUT);
        if (!ok) break;
        issue(g);
        issued = g + 1;
      }
      // Let the copies this CTA started land before it exits: the consumer
      // warps wait for every group too, but one whose wait ran out stops
      // waiting, so the producer confirms the last group of each slot itself
      // (bounded; at once in a normal run).
      for (int g = (issued > NG ? issued - NG : 0); g < issued; ++g)
        mbar_wait_bounded(&full[g % NG], (g / NG) & 1, nullptr, 0);
    }
  } else {

  // per-lane indices inside the staged column windows
  const int n_idx = y - Y0 + 2;
  const int e_idx = y - Y0 + (LEAD - 1 - EWin<T>::OFF);  // element row y-1; row y is +1
  const int m_idx = y + LEAD - ms;

  // Element-centric march. At step c lane y transforms node (c, y) (p_new,
  // or u with fixed DOFs zeroed), forms element (c-1, y) from its corners
  // (c-1, y) (c, y) (c, y+1) (c-1, y+1), and finishes node (c-1, y): the carry
  // holds what elements (c-2, y) and (c-2, y-1) gave it one step earlier.
  const V2<C> zero2 = mk2<C>(C(0), C(0));
  V2<C> pn_prev = zero2, pu_prev = zero2, carry = zero2;
  C sprev_d = C(0), sprev_u = C(0);  // element column c-1, rows y-1, y
  C s2_d = C(0), s2_u = C(0);        // element column c-2, rows y-1, y (residual modes)
  unsigned m_prev = 0;

  for (int k = 0; k < NC; ++k) {
    const int c = cA + k;
    const int g = k / G, kk = k - g * G;
    if (kk == 0 && ok) ok = mbar_wait_bounded(&full[g % NG], (g / NG) & 1, a.err, ERR_TMA_TIMEOUT);
    const unsigned char *sb = smem + (g % NG) * SLOT;
    const V2<T> *colA = reinterpret_cast<const V2<T> *>(sb + kk * Geo::CNB);
    const V2<T> *colB = reinterpret_cast<const V2<T> *>(sb + G * Geo::CNB + kk * Geo::CNB);
    const T *colS = reinterpret_cast<const T *>(sb + G * Geo::CNB * (Geo::HAS_B ? 2 : 1) +
                                                kk * Geo::CEB);
    const uint8_t *colM = sb + G * Geo::CNB * (Geo::HAS_B ? 2 : 1) + G * Geo::CEB + kk * Geo::CMB;
    const bool node_ok = (!SCALE_COL || c > cA) && c >= 0 && c <= nx;
    const bool elem_ok = c >= 0 && c < nx;
    const C scd = elem_ok ? C(colS[e_idx]) : C(0);      // element (c, y-1)
    const C scu = elem_ok ? C(colS[e_idx + 1]) : C(0);  // element (c, y)

    // ---- transformed nodal value at (c, y)
    V2<C> v = zero2;
    const unsigned m = node_ok ? colM[m_idx] : 0u;
    if (node_ok) {
      const V2<C> av = cvt2<C, T>(colA[n_idx]);
      if constexpr (MODE == M_RAW) {
        v = av;
      } else if constexpr (MODE == M_DIR) {
        V2<C> z;
        if constexpr (PRE == TPO_PRECOND_BLOCK_JACOBI) z = av;
        else z = point_precond<C, PRE>(av, m, sprev_d, sprev_u, scd, scu);
        if (first) {
          v = z;
        } else {
          const V2<C> po = cvt2<C, T>(colB[n_idx]);
          v = mk2<C>(fmaT(beta, po.x, z.x), fmaT(beta, po.y, z.y));
        }
        v = cvt2<C, T>(mk2<T>(T(v.x), T(v.y)));  // the stored direction is what K sees
      } else {  // M_RES, M_RESX: u with fixed DOFs zeroed (idempotent write-back)
        v = av;
        if (m & FIXED_X) v.x = C(0);
        if (m & FIXED_Y) v.y = C(0);
        if (m && own_row && c >= x0 && c < x1)
          st2<T>(static_cast<T *>(a.uw), pslot(c, y, P), mk2<T>(T(v.x), T(v.y)));
      }
    }
    const V2<C> vu = shfl_down2<C>(v);  // node (c, y+1)

    // ---- element (c-1, y): corners (c-1,y) (c,y) (c,y+1) (c-1,y+1)
    V2<C> fbl, fbr, ftr, ftl;
    elem_forces<C>(sprev_u, pn_prev, v, vu, pu_prev, fbl, fbr, ftr, ftl);
    const V2<C> tl_below = shfl_up2<C>(ftl);  // element (c-1, y-1) -> node (c-1, y)
    const V2<C> tr_below = shfl_up2<C>(ftr);  // element (c-1, y-1) -> node (c, y)

    // this warp is done with group g: release it; thread 0 then stages
    // group g + NG - 1 into the slot of group g - 1
    if (kk == G - 1 || k == NC - 1) {  // group done: release it to the producer
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[g % NG]);
    }

    // ---- node (xo, y), xo = c - 1, is complete
    const int xo = c - 1;
    if (own_row && xo >= x0) {
      const size_t node = pslot(xo, y, P);
      V2<C> kv = mk2<C>(carry.x + fbl.x + tl_below.x, carry.y + fbl.y + tl_below.y);
      if (m_prev & FIXED_X) kv.x = pn_prev.x;  // identity rows at fixed DOFs
      if (m_prev & FIXED_Y) kv.y = pn_prev.y;
      if constexpr (MODE == M_RAW) {
        const V2<T> ks = mk2<T>(T(kv.x), T(kv.y));
        st2<T>(static_cast<T *>(a.out), node, ks);
        acc[0] += (double)pn_prev.x * (double)ks.x + (double)pn_prev.y * (double)ks.y;
      } else if constexpr (MODE == M_DIR) {
        const V2<T> ks = mk2<T>(T(kv.x), T(kv.y));
        st2<T>(dst_p, node, mk2<T>(T(pn_prev.x), T(pn_prev.y)));
        st2<T>(static_cast<T *>(a.out), node, ks);
        acc[0] += (double)pn_prev.x * (double)ks.x + (double)pn_prev.y * (double)ks.y;
      } else if constexpr (MODE == M_RES) {
        const V2<C> f = cvt2<C, T>(ld2<T>(static_cast<const T *>(a.f), node));
        const V2<T> r = mk2<T>(T(f.x - kv.x), T(f.y - kv.y));
        st2<T>(static_cast<T *>(a.out), node, r);
        if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
          const V2<C> z = point_precond<C, PRE>(cvt2<C, T>(r), m_prev, s2_d, s2_u, sprev_d,
                                                sprev_u);
          acc[0] += (double)r.x * z.x + (double)r.y * z.y;
        }
        acc[1] += (double)r.x * r.x + (double)r.y * r.y;
      } else {  // M_RESX: T == C == double; the inner solve stores float
        const double2 f = ld2<double>(static_cast<const double *>(a.f), node);
        const double rx = f.x - (double)kv.x, ry = f.y - (double)kv.y;
        acc[0] += rx * rx + ry * ry;
        const float2 r32 = make_float2((float)rx, (float)ry);
        st2<float>(static_cast<float *>((a.out2 && (ctl->it & 1)) ? a.out2 : a.out), node, r32);
        if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
          // the inner kernels see FP32-stored scales: use the same here
          const double2 z = point_precond<double, PRE>(
              make_double2(r32.x, r32.y), m_prev, (double)(float)s2_d, (double)(float)s2_u,
              (double)(float)sprev_d, (double)(float)sprev_u);
          acc[1] += (double)r32.x * z.x + (double)r32.y * z.y;
        }
        acc[2] += (double)r32.x * r32.x + (double)r32.y * r32.y;
      }
    }
    carry = mk2<C>(fbr.x + tr_below.x, fbr.y + tr_below.y);
    pn_prev = v;
    pu_prev = vu;
    s2_d = sprev_d;
    s2_u = sprev_u;
    sprev_d = scd;
    sprev_u = scu;
    m_prev = m;
  }

  }  // consumer warps
  __syncthreads();  // no warp leaves while the producer may still be staging
  uint32_t *counter = (MODE == M_RESX) ? &a.octl->counter : &ctl->counter;
  if (!grid_reduce<NV>(acc, a.part, counter, nb, bid)) return;
  if (threadIdx.x != 0) return;
  if constexpr (MODE == M_RAW) {
    if (a.result) *a.result = acc[0];
  } else if constexpr (MODE == M_DIR) {
    const double pap = acc[0];
    ctl->pap = pap;
    ctl->first = 0;
    if (!finite(pap)) ctl->status = TPO_SOLVE_NONFINITE;
    else if (fabs(pap) < 1e-30) ctl->status = TPO_SOLVE_BREAKDOWN;  // solver.py:114-115
    else ctl->alpha = ctl->rz / pap;                                  // solver.py:117
  } else if constexpr (MODE == M_RES) {
    ctl->it = 0;
    ctl->first = 1;
    ctl->rr = acc[1];
    if (PRE != TPO_PRECOND_BLOCK_JACOBI) ctl->rz = acc[0];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  } else {
    // FP64 residual of the mixed form: first residual of the solve, or a
    // replacement of the inner recursive residual ("reliable update")
    OuterCtl *o = a.octl;
    o->rr = acc[0];
    o->it += 1;
    const bool cont = o->it > 1;
    if (!finite(acc[0]) || !finite(acc[1]) || !finite(acc[2])) o->status = TPO_SOLVE_NONFINITE;
    else if (acc[0] < o->tol_sq) o->status = TPO_SOLVE_CONVERGED;
    else if (o->it > o->max_outer) o->status = TPO_SOLVE_MAX_ITER;
    ctl->rmax2 = acc[0];
    ctl->since = 0;
    ctl->rr = acc[2];
    ctl->cont = cont ? 1 : 0;
    if (PRE != TPO_PRECOND_BLOCK_JACOBI) {
      if (cont) {
        ctl->beta = acc[1] / (ctl->rz + 1e-60);  // keep the direction
        ctl->first = 0;
      } else {
        ctl->first = 1;
      }
      ctl->rz = acc[1];
    }
    ctl->status = o->status;  // RUNNING, or the outer solve's end state
  }
}

template <typename T, typename C, int MODE, int PRE, int G, int NG>
__global__ void __launch_bounds__(TS_THREADS) k_tstencil(TsArgs a, int L) {
  tstencil_run<T, C, MODE, PRE, G, NG>(a, L, blockIdx.x, blockIdx.y, gridDim.x * gridDim.y,
                                       blockIdx.y * gridDim.x + blockIdx.x);
}

// ---------------------------------------------------------------------------
// PCG update (pointwise): u += alpha p, r -= alpha Ap, z = M r, r.z, ||r||^2,
// then the stop / replacement / beta logic of the step's last CTA.
// ---------------------------------------------------------------------------
struct UpdArgs {
  int nx, ny, P;
  const void *s;
  const uint8_t *mask;
  void *u, *r;
  const void *ap;
  const void *pa, *pb;
  double *part;
  PcgCtl *ctl;
  void *z;  // flat update: optional output z = M r (T), read by the next direction kernel
};

__device__ __forceinline__ void finish_update(PcgCtl *ctl, double rz_new, double rr) {
  ctl->it += 1;
  ctl->rr = rr;
  if (!finite(rz_new) || !finite(rr)) {
    ctl->status = TPO_SOLVE_NONFINITE;
    return;
  }
  if (ctl->rupd2 > 0.0) {
    // mixed form: the recursive FP32 residual only schedules an FP64
    // residual replacement (when it has dropped by inner_tol below the
    // largest residual seen since the last replacement, or every
    // kReplaceEvery iterations); convergence is decided on the FP64 residual
    ctl->rmax2 = fmax(ctl->rmax2, rr);
    ctl->since += 1;
    if (rr < ctl->rupd2 * ctl->rmax2 || rr < ctl->tol_sq || ctl->since >= kReplaceEvery) {
      ctl->status = SOLVE_NEED_UPDATE;
      return;
    }
  } else if (rr < ctl->tol_sq) {  // reference solver.py:147-149
    ctl->status = TPO_SOLVE_CONVERGED;
    return;
  }
  if (ctl->it >= ctl->max_iter) {
    ctl->status = TPO_SOLVE_MAX_ITER;
    return;
  }
  ctl->beta = rz_new / (ctl->rz + 1e-60);  // solver.py:151
  ctl->rz = rz_new;
}


// Same update, pointwise over the grid's nodes with a flat grid-stride loop.
// A warp takes runs of RUN = 32 UQ consecutive grid nodes (the compact
// numbering, column after column); lane l holds nodes base + l + 32 j,
// j < UQ, so every load and store instruction of the warp covers 32
// consecutive nodes (one break per column boundary), and all UQ nodes' loads
// are issued before any is used. The node's four element scales come
// straight from the padded scale array: element (c-1, y-1), (c-1, y),
// (c, y-1), (c, y) sit at the node's slot - P - 1, - P, - 1 and + 0 (zero
// pads outside the grid rows).
constexpr int UF_THREADS = 256;
#ifndef TPO_UQ
#define TPO_UQ 1
#endif
constexpr int UQ = TPO_UQ;  // nodes per lane and pass
constexpr int RUN = 32 * UQ;

// n / d for 0 <= n < 2^31 through a double reciprocal, corrected to exact
__device__ __forceinline__ int div_exact(int n, int d, double inv_d) {
  int q = (int)((double)n * inv_d);
  if ((q + 1) * d <= n) ++q;
  if (q * d > n) --q;
  return q;
}

template <typename T, typename C, typename X> struct FlatNode {
  size_t slot;
  V2<X> u;
  V2<T> r, p, ap;
  C s_ll, s_lh, s_rl, s_rh;
  unsigned m;
  bool ok;
};

// loads of grid node n (compact numbering) for the flat kernels; UPD also
// loads u, p and Ap (the update), otherwise only r
template <typename T, typename C, typename X, bool SCALES, bool UPD>
__device__ __forceinline__ void flat_load(FlatNode<T, C, X> &d, int n, int total, int ny1,
                                          double inv, int nx, int P, const X *__restrict__ u,
                                          const T *__restrict__ r, const T *__restrict__ p,
                                          const T *__restrict__ ap, const T *__restrict__ s,
                                          const uint8_t *__restrict__ mask) {
  d.ok = n < total;
  d.s_ll = d.s_lh = d.s_rl = d.s_rh = C(0);
  if (!d.ok) return;
  const int c = div_exact(n, ny1, inv), y = n - c * ny1;
  d.slot = (size_t)c * P + y + LEAD;
  d.r = ld2<T>(r, d.slot);
  if constexpr (UPD) {
    d.u = ld2<X>(u, d.slot);
    d.p = ld2<T>(p, d.slot);
    d.ap = ld2<T>(ap, d.slot);
  }
  d.m = mask[d.slot];
  if constexpr (SCALES) {
    if (c >= 1) {
      d.s_ll = C(s[d.slot - P - 1]);
      d.s_lh = C(s[d.slot - P]);
    }
    if (c < nx) {
      d.s_rl = C(s[d.slot - 1]);
      d.s_rh = C(s[d.slot]);
    }
  }
}

template <typename T, typename C, int PRE, typename X = T>
__device__ __forceinline__ void update_flat_run(const UpdArgs &a, int bx, int gx, int nb,
                                                int bid) {
  PcgCtl *ctl = a.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const double alpha = ctl->alpha;
  const C alpha_c = C(alpha);
  const T *__restrict__ p = static_cast<const T *>((ctl->it & 1) ? a.pa : a.pb);
  const int nx = a.nx, ny1 = a.ny + 1, P = a.P;
  const double inv = 1.0 / ny1;
  const T *__restrict__ s = static_cast<const T *>(a.s);
  X *__restrict__ u = static_cast<X *>(a.u);
  T *__restrict__ r = static_cast<T *>(a.r);
  T *__restrict__ zo = static_cast<T *>(a.z);
  const T *__restrict__ ap = static_cast<const T *>(a.ap);
  const uint8_t *__restrict__ mask = a.mask;
  const int total = (nx + 1) * ny1;
  const int lane = threadIdx.x & 31;
  const int warp = (bx * blockDim.x + threadIdx.x) >> 5, nwarps = (gx * blockDim.x) >> 5;
  double acc[2] = {0.0, 0.0};
  for (int base = warp * RUN; base < total; base += nwarps * RUN) {
    FlatNode<T, C, X> d[UQ];
#pragma unroll
    for (int j = 0; j < UQ; ++j)
      flat_load<T, C, X, PRE != TPO_PRECOND_NONE, true>(d[j], base + 32 * j + lane, total, ny1,
                                                         inv, nx, P, u, r, p, ap, s, mask);
#pragma unroll
    for (int j = 0; j < UQ; ++j) {
      if (!d[j].ok) continue;
      // the solution accumulates in FP64 in every form
      const V2<X> un = mk2<X>(X(fma(alpha, (double)d[j].p.x, (double)d[j].u.x)),
                              X(fma(alpha, (double)d[j].p.y, (double)d[j].u.y)));
      const V2<T> rn = mk2<T>(T(fmaT(-alpha_c, C(d[j].ap.x), C(d[j].r.x))),
                              T(fmaT(-alpha_c, C(d[j].ap.y), C(d[j].r.y))));
      st2<X>(u, d[j].slot, un);
      st2<T>(r, d[j].slot, rn);
      C pa, pb, pd;
      node_pre<C, PRE>(d[j].m, d[j].s_ll, d[j].s_lh, d[j].s_rl, d[j].s_rh, pa, pb, pd);
      const V2<C> z = pre_apply<C>(pa, pb, pd, cvt2<C, T>(rn));
      if (zo) {  // r.z with the stored (rounded) z, the one the direction update uses
        const V2<T> zt = mk2<T>(T(z.x), T(z.y));
        st2<T>(zo, d[j].slot, zt);
        acc[0] += dot2d(rn, zt);
      } else {
        acc[0] += dot2d(rn, z);
      }
      acc[1] += dot2d(rn, rn);
    }
  }
  if (!grid_reduce<2>(acc, a.part, &ctl->counter, nb, bid)) return;
  if (threadIdx.x == 0) finish_update(ctl, acc[0], acc[1]);
}

// z = M r over the grid's nodes (flat), after an FP64 residual replacement:
// the direction kernel reads z instead of recomputing it
template <typename T, typename C, int PRE>
__device__ __forceinline__ void precond_flat_run(int nx, int ny, int P, const T *__restrict__ s,
                                                 const uint8_t *__restrict__ mask,
                                                 const T *__restrict__ r, T *__restrict__ z,
                                                 int bx, int gx) {
  const int ny1 = ny + 1;
  const double inv = 1.0 / ny1;
  const int total = (nx + 1) * ny1;
  const int lane = threadIdx.x & 31;
  const int warp = (bx * blockDim.x + threadIdx.x) >> 5, nwarps = (gx * blockDim.x) >> 5;
  for (int base = warp * RUN; base < total; base += nwarps * RUN) {
    FlatNode<T, C, T> d[UQ];
#pragma unroll
    for (int j = 0; j < UQ; ++j)
      flat_load<T, C, T, PRE != TPO_PRECOND_NONE, false>(d[j], base + 32 * j + lane, total, ny1,
                                                          inv, nx, P, nullptr, r, nullptr,
                                                          nullptr, s, mask);
#pragma unroll
    for (int j = 0; j < UQ; ++j) {
      if (!d[j].ok) continue;
      C pa, pb, pd;
      node_pre<C, PRE>(d[j].m, d[j].s_ll, d[j].s_lh, d[j].s_rl, d[j].s_rh, pa, pb, pd);
      const V2<C> zz = pre_apply<C>(pa, pb, pd, cvt2<C, T>(d[j].r));
      st2<T>(z, d[j].slot, mk2<T>(T(zz.x), T(zz.y)));
    }
  }
}
template <typename T, typename C, int PRE>
__global__ void __launch_bounds__(UF_THREADS) k_precond_flat(int nx, int ny, int P, const T *s,
                                                             const uint8_t *mask, const T *r,
                                                             T *z) {
  precond_flat_run<T, C, PRE>(nx, ny, P, s, mask, r, z, blockIdx.x, gridDim.x);
}

// the same pass, run only right after an FP64 residual replacement of the
// mixed form (ctl->since == 0) while the solve goes on: the device-side loop
// of tpo_pcg_solve_async enqueues it every loop body
template <typename T, typename C, int PRE>
__global__ void __launch_bounds__(UF_THREADS) k_precond_gated(const PcgCtl *ctl, int nx, int ny,
                                                              int P, const T *s,
                                                              const uint8_t *mask, const T *r,
                                                              T *z) {
  if (ctl->status != TPO_SOLVE_RUNNING || ctl->since != 0) return;
  precond_flat_run<T, C, PRE>(nx, ny, P, s, mask, r, z, blockIdx.x, gridDim.x);
}

template <typename T, typename C, int PRE, typename X = T>
__global__ void __launch_bounds__(UF_THREADS) k_update_flat(UpdArgs a) {
  update_flat_run<T, C, PRE, X>(a, blockIdx.x, gridDim.x, gridDim.x, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Element-block preconditioner (the reference's "block_jacobi",
// fem/preconditioner.py:47-108):
//   z = C^-1/2 sum_e w_e Ke_inv (C^-1/2 r)_e,  w_e = s_e / max(s_e, alpha)^2,
//   z[fixed] = 0,  C = elements per node.
// UPDATE: r_new = r - alpha Ap is formed for the strip and its halo (read from
// one residual buffer, written to the other), u += alpha p on owned nodes,
// then z from r_new, and the convergence/beta logic.
// INIT:   z from r as it is (first residual of a solve, or a replaced one).
// ---------------------------------------------------------------------------
struct BlkArgs {
  int nx, ny, P;
  const void *w;
  const uint8_t *mask;
  void *u;
  const void *ap;
  const void *pa, *pb;
  void *ra, *rb;
  void *z;
  double *part;
  PcgCtl *ctl;
  int gate;  // INIT: run only right after a residual evaluation (ctl->since == 0)
};

template <typename T, typename C, bool INIT, int L, typename X = T>
__global__ void __launch_bounds__(ST_THREADS) k_blockpre(BlkArgs a) {
  PcgCtl *ctl = a.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  if (INIT && a.gate && ctl->since != 0) return;  // no replacement since the last INIT
  const int parity = ctl->it & 1;
  const C alpha = INIT ? C(0) : C(ctl->alpha);
  const T *r_src = static_cast<const T *>(parity ? a.rb : a.ra);
  T *r_dst = static_cast<T *>(parity ? a.ra : a.rb);
  const T *__restrict__ p = static_cast<const T *>(parity ? a.pa : a.pb);
  const int nx = a.nx, ny = a.ny, P = a.P;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int y = gw * RPW - 1 + lane;
  const bool row_ok = (y >= 0) && (y <= ny);
  const bool own_row = row_ok && lane >= 1 && lane <= RPW;
  const int x0 = blockIdx.y * L;
  const int x1 = min(x0 + L, nx + 1);
  const T *__restrict__ w = static_cast<const T *>(a.w);
  X *__restrict__ u = static_cast<X *>(a.u);
  const T *__restrict__ ap = static_cast<const T *>(a.ap);
  T *__restrict__ z = static_cast<T *>(a.z);

  C e0d = C(0), e0u = C(0), e1d = C(0), e1u = C(0);
  const V2<C> zero2 = mk2<C>(C(0), C(0));
  V2<C> n0d = zero2, n0m = zero2, n0u = zero2, n1d = zero2, n1m = zero2, n1u = zero2;
  V2<C> n2d = zero2, n2m = zero2, n2u = zero2;
  V2<C> rn1 = zero2, rn2 = zero2;  // unscaled residual at columns c-1, c
  unsigned m1 = 0, m2 = 0;
  double acc[2] = {0.0, 0.0};

  struct Raw {
    C wd, wu;
    V2<T> r, ap, p;
    V2<X> u;
    unsigned m;
  };
  const V2<T> tz = mk2<T>(T(0), T(0));
  auto fetch = [&](int c, Raw &R) {
    R.wd = R.wu = C(0);
    const int ce = c - 1;
    if (ce >= 0 && ce < nx && row_ok) {
      const size_t e = pslot(ce, y, P);
      R.wd = C(w[e - 1]);
      R.wu = C(w[e]);
    }
    R.m = 0;
    R.r = R.ap = R.p = tz;
    R.u = mk2<X>(X(0), X(0));
    if (row_ok && c >= 0 && c <= nx) {
      const size_t node = pslot(c, y, P);
      R.m = a.mask[node];
      R.r = ld2<T>(r_src, node);
      if (!INIT) {
        R.ap = ld2<T>(ap, node);
        if (own_row && c >= x0 && c < x1) {
          R.u = ld2<X>(u, node);
          R.p = ld2<T>(p, node);
        }
      }
    }
  };
  Raw nxt;
  fetch(x0 - 1, nxt);
  for (int c = x0 - 1; c <= x1; ++c) {
    const Raw cur = nxt;
    if (c < x1) fetch(c + 1, nxt);
    e0d = e1d; e0u = e1u;
    e1d = cur.wd;
    e1u = cur.wu;
    V2<C> rt = zero2, rn = zero2;
    const unsigned m = cur.m;
    if (row_ok && c >= 0 && c <= nx) {
      const size_t node = pslot(c, y, P);
      rn = cvt2<C, T>(cur.r);
      if (!INIT) {
        const V2<T> rs = mk2<T>(T(fmaT(-alpha, C(cur.ap.x), rn.x)),
                                T(fmaT(-alpha, C(cur.ap.y), rn.y)));
        rn = cvt2<C, T>(rs);
        if (own_row && c >= x0 && c < x1) {
          // the solution accumulates in FP64 in every form
          const double al = ctl->alpha;
          st2<X>(u, node, mk2<X>(X(fma(al, (double)cur.p.x, (double)cur.u.x)),
                                 X(fma(al, (double)cur.p.y, (double)cur.u.y))));
          st2<T>(r_dst, node, rs);
        }
      }
      const C sq = sqrt(C(node_elem_count(c, y, nx, ny)));
      rt = mk2<C>(rn.x / sq, rn.y / sq);
    }
    n0d = n1d; n0m = n1m; n0u = n1u;
    n1d = n2d; n1m = n2m; n1u = n2u;
    rn1 = rn2; rn2 = rn;
    m1 = m2; m2 = m;
    n2m = rt;
    n2d = shfl_up2<C>(rt);
    n2u = shfl_down2<C>(rt);

    const int xo = c - 1;
    if (own_row && xo >= x0) {
      const size_t node = pslot(xo, y, P);
      V2<C> zz = node_apply<C, true>(n0d, n0m, n0u, n1d, n1m, n1u, n2d, n2m, n2u, e0d, e0u, e1d,
                                     e1u);
      const C sq = sqrt(C(node_elem_count(xo, y, nx, ny)));
      const V2<T> zs = mk2<T>((m1 & FIXED_X) ? T(0) : T(zz.x / sq),
                              (m1 & FIXED_Y) ? T(0) : T(zz.y / sq));
      st2<T>(z, node, zs);
      acc[0] += (double)rn1.x * (double)zs.x + (double)rn1.y * (double)zs.y;
      acc[1] += (double)rn1.x * rn1.x + (double)rn1.y * rn1.y;
    }
  }
  if (!grid_reduce<2>(acc, a.part, &ctl->counter)) return;
  if (threadIdx.x != 0) return;
  if (INIT) {
    // first residual of a solve, or (mixed form) a replaced residual
    if (ctl->cont) {
      ctl->beta = acc[0] / (ctl->rz + 1e-60);
      ctl->first = 0;
    } else {
      ctl->first = 1;
    }
    ctl->rz = acc[0];
    ctl->rr = acc[1];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  } else {
    finish_update(ctl, acc[0], acc[1]);
  }
}

// ---------------------------------------------------------------------------
// Per-solve setup and small helpers (padded layout)
// ---------------------------------------------------------------------------
// s = e_min + rho^p (1 - e_min) (reference fem/kernels.py:92), its FP32 copy,
// and the element-block weights w = s / max(s, alpha)^2 (preconditioner.py:55-57).
// Writes every slot of the padded arrays (pads = 0).
__device__ __forceinline__ void scales_run(int nx, int ny, int P, const double *__restrict__ rho,
                                           double e_min, double pen, double alpha_reg,
                                           double *__restrict__ s64, float *__restrict__ s32,
                                           double *__restrict__ w64, float *__restrict__ w32,
                                           int bx, int gx) {
  const size_t total = (size_t)nx * P;
  for (size_t i = bx * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gx * blockDim.x) {
    const int ex = (int)(i / P), ey = (int)(i % P) - LEAD;
    double s = 0.0, w = 0.0;
    if (ey >= 0 && ey < ny) {
      s = e_min + pow(rho[(size_t)ex * ny + ey], pen) * (1.0 - e_min);
      const double sc = fmax(s, alpha_reg);
      w = s / (sc * sc);
    }
    if (s64) s64[i] = s;
    if (s32) s32[i] = (float)s;
    if (w64) w64[i] = w;
    if (w32) w32[i] = (float)w;
  }
}
__global__ void k_scales(int nx, int ny, int P, const double *__restrict__ rho, double e_min,
                         double pen, double alpha_reg, double *__restrict__ s64,
                         float *__restrict__ s32, double *__restrict__ w64,
                         float *__restrict__ w32) {
  scales_run(nx, ny, P, rho, e_min, pen, alpha_reg, s64, s32, w64, w32, blockIdx.x, gridDim.x);
}

// element values (compact, T) -> SIMP scales, padded T
template <typename T>
__global__ void k_scales_t(int nx, int ny, int P, const T *__restrict__ rho, double e_min,
                           double pen, T *__restrict__ s) {
  const size_t total = (size_t)nx * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int ex = (int)(i / P), ey = (int)(i % P) - LEAD;
    s[i] = (ey >= 0 && ey < ny)
               ? T(e_min + pow((double)rho[(size_t)ex * ny + ey], pen) * (1.0 - e_min))
               : T(0);
  }
}

// precomputed compact scales -> padded
template <typename T>
__global__ void k_pad_elems(int nx, int ny, int P, const T *__restrict__ src, T *__restrict__ dst) {
  const size_t total = (size_t)nx * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int ex = (int)(i / P), ey = (int)(i % P) - LEAD;
    dst[i] = (ey >= 0 && ey < ny) ? src[(size_t)ex * ny + ey] : T(0);
  }
}

// Per-solve control state. The mixed form (octl non-null) starts in
// SOLVE_NEED_UPDATE: its first step is the FP64 residual.
__device__ __forceinline__ void ctl_init_run(PcgCtl *ctl, double tol_sq, double rupd2,
                                             int max_iter, OuterCtl *octl, double outer_tol_sq,
                                             int max_outer) {
  ctl->rz = 0.0;
  ctl->alpha = 0.0;
  ctl->beta = 0.0;
  ctl->rr = 0.0;
  ctl->pap = 0.0;
  ctl->tol_sq = tol_sq;
  ctl->rupd2 = rupd2;
  ctl->rmax2 = 0.0;
  ctl->it = 0;
  ctl->status = octl ? SOLVE_NEED_UPDATE : TPO_SOLVE_RUNNING;
  ctl->max_iter = max_iter;
  ctl->first = 1;
  ctl->cont = 0;
  ctl->since = 0;
  ctl->phase = 0;
  ctl->err = 0;
  ctl->counter = 0u;
  if (octl) {
    octl->rr = 0.0;
    octl->tol_sq = outer_tol_sq;
    octl->it = 0;
    octl->status = TPO_SOLVE_RUNNING;
    octl->counter = 0u;
    octl->max_outer = max_outer;
  }
}
__global__ void k_ctl_init(PcgCtl *ctl, double tol_sq, double rupd2, int max_iter,
                           OuterCtl *octl, double outer_tol_sq, int max_outer) {
  ctl_init_run(ctl, tol_sq, rupd2, max_iter, octl, outer_tol_sq, max_outer);
}


}  // namespace tpo
