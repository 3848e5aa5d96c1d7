// One PCG iteration per launch, for the point preconditioners (Jacobi, 2x2
// nodal block-Jacobi, none).
//
// The reference's PCG (fem/solver.py:27-159) needs two global reductions per
// iteration (p.Ap, then r.z), which costs two launches here. This kernel runs
// the Chronopoulos-Gear form of the same preconditioned CG, which needs one:
// with u = M^-1 r and w = K u kept as vectors,
//   p_i     = u_i + beta_i p_{i-1}          s_i = w_i + beta_i s_{i-1}  (= K p_i)
//   x_{i+1} = x_i + alpha_i p_i             r_{i+1} = r_i - alpha_i s_i
//   u_{i+1} = M^-1 r_{i+1}                  w_{i+1} = K u_{i+1}
//   gamma = r.u, delta = w.u, ||r||^2       (one reduction)
//   beta_{i+1} = gamma_{i+1} / gamma_i,  p.Kp = delta - beta_{i+1} gamma_{i+1} / alpha_i,
//   alpha_{i+1} = gamma_{i+1} / p.Kp.
// In exact arithmetic the iterates equal the reference's. The stop test
// (||r||^2 < tol^2 ||f||^2 on the recursive residual, after the update), the
// breakdown test (|p.Kp| < 1e-30) and beta = gamma_new / (gamma_old + 1e-60)
// follow the reference.
//
// Layout and pipeline are those of k_tstencil (layout.cuh): a CTA owns 120
// rows and a strip of L node columns. Every input is staged per column by
// cp.async.bulk into an mbarrier ring: r, w, s (needed around a node by the
// stencil), p and x (pointwise; owned columns only), the element scales and
// the fixed mask. r, w and s ping-pong between two buffers (strips read their
// neighbours' columns); p and x are updated in place by their owner only.
//
// INIT launch (ctl->first = 1): alpha = beta = 0. It forms u = M^-1 r and
// w = K u for the first residual, p = u, and gamma, delta, ||r||^2, from which
// the last CTA sets alpha = gamma / delta.
//
// FP64 storage only. With FP32-stored vectors the recurrence s = w + beta s
// drifts away from K p, and p.Kp, formed from sums rather than from a fresh
// K p, loses its accuracy; the mixed form therefore keeps the two-launch
// recurrence, which recomputes K p every iteration.
#pragma once

#include "common.cuh"
#include "layout.cuh"
#include "stencil.cuh"
#include "pcg.cuh"  // ST_THREADS, ERR_TMA_TIMEOUT, cvt2

namespace tpo {

struct CgArgs {
  int nx, ny, P;
  const void *s;          // element scales (T, padded)
  const uint8_t *mask;    // fixed mask (padded)
  void *ra, *rb;          // residual ping-pong
  void *wa, *wb;          // w = K M^-1 r ping-pong
  void *sa, *sb;          // s = K p ping-pong
  void *p;                // direction (in place)
  void *x;                // solution u
  double *part;
  PcgCtl *ctl;
  int *err;
};

template <typename T> struct CgGeom {
  static constexpr int CNB = N_WIN * 2 * (int)sizeof(T);   // node bytes per column and vector
  static constexpr int CEB = EWin<T>::N * (int)sizeof(T);  // element-scale bytes per column
  static constexpr int CMB = M_WIN;                        // mask bytes per column
  // slot: r, w, s, p, x (node windows), scales, mask
  static constexpr int OFF_E = 5 * CNB, OFF_M = OFF_E + CEB, SLOT = OFF_M + CMB;
};

// 4 consumer warps (120 grid rows) and one producer warp that only stages
// columns, so refills never wait for a consumer warp's arithmetic
constexpr int CG_THREADS = (WPC + 1) * 32;

template <typename T, typename C, int PRE, int NG>
__global__ void __launch_bounds__(CG_THREADS) k_cgstep(CgArgs A, int L) {
  using Geo = CgGeom<T>;
  constexpr int SLOT = Geo::SLOT;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[NG];   // column staged (TMA transaction bytes)
  __shared__ __align__(8) uint64_t empty[NG];  // column consumed by all warps

  PcgCtl *ctl = A.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const bool init = ctl->first != 0;
  const C alpha = init ? C(0) : C(ctl->alpha);
  const C beta = init ? C(0) : C(ctl->beta);
  const int par = ctl->phase & 1;
  const T *r_in = static_cast<const T *>(par ? A.rb : A.ra);
  const T *w_in = static_cast<const T *>(par ? A.wb : A.wa);
  const T *s_in = static_cast<const T *>(par ? A.sb : A.sa);
  T *r_out = static_cast<T *>(par ? A.ra : A.rb);
  T *w_out = static_cast<T *>(par ? A.wa : A.wb);
  T *s_out = static_cast<T *>(par ? A.sa : A.sb);
  T *pv = static_cast<T *>(A.p);
  T *xv = static_cast<T *>(A.x);
  const T *gs = static_cast<const T *>(A.s);

  const int nx = A.nx, ny = A.ny, P = A.P;
  const int Y0 = blockIdx.x * RPC;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int y = Y0 + wid * RPW - 1 + lane;
  const bool own_row = lane >= 1 && lane <= RPW && y <= ny;
  const int x0 = blockIdx.y * L;
  const int x1 = min(x0 + L, nx + 1);
  const int cA = x0 - 2;       // first staged column (element scales only)
  const int NC = x1 - cA + 1;  // staged columns cA..x1
  const int ms = (Y0 + LEAD - 1) & ~15;

  // producer (lane 0 of warp WPC): stage column cA + k into ring slot k % NG,
  // after the column that used the slot before (k - NG) has been released by
  // every consumer warp
  auto issue = [&](int k) {
    unsigned char *sb = smem + (k % NG) * SLOT;
    uint64_t *bar = &full[k % NG];
    const int c = cA + k;
    const bool node_ok = c > cA && c >= 0 && c <= nx;
    const bool own = c >= x0 && c < x1;
    const bool elem_ok = c >= 0 && c < nx;
    const unsigned bytes = (node_ok ? 3 * Geo::CNB + Geo::CMB : 0) +
                           (own ? (init ? 1 : 2) * Geo::CNB : 0) + (elem_ok ? Geo::CEB : 0);
    mbar_arrive_expect_tx(bar, bytes);
    const size_t col = 2 * ((size_t)c * P + Y0 + N_OFF);
    if (node_ok) {
      bulk_g2s(sb, r_in + col, Geo::CNB, bar);
      bulk_g2s(sb + Geo::CNB, w_in + col, Geo::CNB, bar);
      bulk_g2s(sb + 2 * Geo::CNB, s_in + col, Geo::CNB, bar);
      bulk_g2s(sb + Geo::OFF_M, A.mask + (size_t)c * P + ms, Geo::CMB, bar);
    }
    if (own) {
      bulk_g2s(sb + 3 * Geo::CNB, pv + col, Geo::CNB, bar);
      if (!init) bulk_g2s(sb + 4 * Geo::CNB, xv + col, Geo::CNB, bar);
    }
    if (elem_ok) bulk_g2s(sb + Geo::OFF_E, gs + (size_t)c * P + Y0 + EWin<T>::OFF, Geo::CEB, bar);
  };
  bool ok = true;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NG; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], WPC);
    }
    fence_mbar_init();
  }
  __syncthreads();
  double acc[3] = {0.0, 0.0, 0.0};  // gamma = r.u, delta = w.u, ||r||^2

  if (wid == WPC) {
    // ---- producer warp
    if (lane == 0) {
      int issued = 0;
      for (int k = 0; k < NC; ++k) {
        if (k >= NG)
          ok = mbar_wait_bounded(&empty[k % NG], ((k / NG) - 1) & 1, A.err, ERR_TMA_TIMEOUT);
        if (!ok) break;  // a consumer stopped releasing: issue nothing more
        issue(k);
        issued = k + 1;
      }
      // let the copies this CTA started land before it exits (the consumers
      // wait for every column too, but one whose wait ran out stops waiting)
      for (int k = (issued > NG ? issued - NG : 0); k < issued; ++k)
        mbar_wait_bounded(&full[k % NG], (k / NG) & 1, nullptr, 0);
    }
  } else {

  const int n_idx = y - Y0 + 2;
  const int e_idx = y - Y0 + (LEAD - 1 - EWin<T>::OFF);  // element row y-1; row y is +1
  const int m_idx = y + LEAD - ms;
  auto own_col = [&](int c) { return own_row && c >= x0 && c < x1; };
  auto slot_of = [&](int c) { return (size_t)c * P + y + LEAD; };

  const V2<C> zero2 = mk2<C>(C(0), C(0));
  const V2<T> zt = mk2<T>(T(0), T(0));
  V2<C> un_prev = zero2, uu_prev = zero2, carry = zero2;
  C sprev_d = C(0), sprev_u = C(0);  // element column c-1, rows y-1, y
  unsigned m_prev = 0;

  for (int k = 0; k < NC; ++k) {
    const int c = cA + k;
    if (ok) ok = mbar_wait_bounded(&full[k % NG], (k / NG) & 1, A.err, ERR_TMA_TIMEOUT);
    const unsigned char *sb = smem + (k % NG) * SLOT;
    const V2<T> *colR = reinterpret_cast<const V2<T> *>(sb);
    const V2<T> *colW = reinterpret_cast<const V2<T> *>(sb + Geo::CNB);
    const V2<T> *colS = reinterpret_cast<const V2<T> *>(sb + 2 * Geo::CNB);
    const V2<T> *colP = reinterpret_cast<const V2<T> *>(sb + 3 * Geo::CNB);
    const V2<T> *colX = reinterpret_cast<const V2<T> *>(sb + 4 * Geo::CNB);
    const T *colE = reinterpret_cast<const T *>(sb + Geo::OFF_E);
    const uint8_t *colM = sb + Geo::OFF_M;
    const bool node_ok = c > cA && c >= 0 && c <= nx;
    const bool elem_ok = c >= 0 && c < nx;
    const C scd = elem_ok ? C(colE[e_idx]) : C(0);      // element (c, y-1)
    const C scu = elem_ok ? C(colE[e_idx + 1]) : C(0);  // element (c, y)

    // ---- node (c, y): s, r updated; u = M^-1 r of the new residual
    V2<C> un = zero2;
    const unsigned m = node_ok ? colM[m_idx] : 0u;
    if (node_ok) {
      const V2<C> rv = cvt2<C, T>(colR[n_idx]);
      const V2<C> wv = cvt2<C, T>(colW[n_idx]);
      const V2<C> sv = cvt2<C, T>(colS[n_idx]);
      C pa, pb, pd;
      node_pre<C, PRE>(m, sprev_d, sprev_u, scd, scu, pa, pb, pd);
      V2<T> s_new, r_new;
      if (init) {
        s_new = zt;
        r_new = colR[n_idx];
      } else {
        s_new = mk2<T>(T(fmaT(beta, sv.x, wv.x)), T(fmaT(beta, sv.y, wv.y)));
        r_new = mk2<T>(T(fmaT(-alpha, C(s_new.x), rv.x)), T(fmaT(-alpha, C(s_new.y), rv.y)));
      }
      const V2<C> rc = cvt2<C, T>(r_new);
      un = pre_apply<C>(pa, pb, pd, rc);
      if (own_col(c)) {
        const size_t o = slot_of(c);
        st2<T>(r_out, o, r_new);
        st2<T>(s_out, o, s_new);
        if (!init) {
          const V2<T> p_cur = colP[n_idx], x_cur = colX[n_idx];
          const V2<C> uo = pre_apply<C>(pa, pb, pd, rv);
          const V2<T> pn = mk2<T>(T(fmaT(beta, C(p_cur.x), uo.x)), T(fmaT(beta, C(p_cur.y), uo.y)));
          st2<T>(pv, o, pn);
          st2<T>(xv, o, mk2<T>(T(fmaT(alpha, C(pn.x), C(x_cur.x))),
                               T(fmaT(alpha, C(pn.y), C(x_cur.y)))));
        } else {
          st2<T>(pv, o, mk2<T>(T(un.x), T(un.y)));  // p_0 = u_0
        }
        acc[0] += (double)rc.x * un.x + (double)rc.y * un.y;
        acc[2] += (double)rc.x * rc.x + (double)rc.y * rc.y;
      }
    }
    const V2<C> uu = shfl_down2<C>(un);  // u at (c, y+1)

    // ---- element (c-1, y): corners (c-1,y) (c,y) (c,y+1) (c-1,y+1)
    V2<C> fbl, fbr, ftr, ftl;
    elem_forces<C>(sprev_u, un_prev, un, uu, uu_prev, fbl, fbr, ftr, ftl);
    const V2<C> tl_below = shfl_up2<C>(ftl);  // element (c-1, y-1) -> node (c-1, y)
    const V2<C> tr_below = shfl_up2<C>(ftr);  // element (c-1, y-1) -> node (c, y)

    // release the column to the producer
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[k % NG]);

    // ---- w = K u at node (c-1, y) is complete
    const int xo = c - 1;
    if (own_row && xo >= x0) {
      V2<C> wv = mk2<C>(carry.x + fbl.x + tl_below.x, carry.y + fbl.y + tl_below.y);
      if (m_prev & FIXED_X) wv.x = un_prev.x;  // identity rows at fixed DOFs
      if (m_prev & FIXED_Y) wv.y = un_prev.y;
      const V2<T> wt = mk2<T>(T(wv.x), T(wv.y));
      st2<T>(w_out, slot_of(xo), wt);
      acc[1] += (double)un_prev.x * (double)wt.x + (double)un_prev.y * (double)wt.y;
    }
    carry = mk2<C>(fbr.x + tr_below.x, fbr.y + tr_below.y);
    un_prev = un;
    uu_prev = uu;
    sprev_d = scd;
    sprev_u = scu;
    m_prev = m;
  }
  }  // consumer warps
  __syncthreads();

  if (!grid_reduce<3>(acc, A.part, &ctl->counter)) return;
  if (threadIdx.x != 0) return;
  const double gamma = acc[0], delta = acc[1], rr = acc[2];
  ctl->phase += 1;
  ctl->rr = rr;
  if (!finite(gamma) || !finite(delta) || !finite(rr)) {
    ctl->status = TPO_SOLVE_NONFINITE;
    return;
  }
  if (!init) {
    ctl->it += 1;
    if (rr < ctl->tol_sq) {  // reference solver.py:147-149
      ctl->status = TPO_SOLVE_CONVERGED;
      return;
    }
    if (ctl->it >= ctl->max_iter) {
      ctl->status = TPO_SOLVE_MAX_ITER;
      return;
    }
  }
  double b = 0.0, pap = delta;
  if (!init) {
    b = gamma / (ctl->rz + 1e-60);          // solver.py:151
    pap = delta - b * gamma / ctl->alpha;   // p_{i+1}.K p_{i+1}
  }
  ctl->pap = pap;
  if (fabs(pap) < 1e-30) {  // solver.py:114-115
    ctl->status = TPO_SOLVE_BREAKDOWN;
    return;
  }
  ctl->alpha = gamma / pap;
  ctl->beta = b;
  ctl->rz = gamma;
  ctl->first = 0;
}

}  // namespace tpo
