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
// the plain FP64 solve, <float,float,double> for the mixed form (FP32 bytes
// and FP32 arithmetic for the matvec, the preconditioner and the vector
// updates; FP64 for the dot products, alpha/beta and the solution). u stays
// FP64 in the mixed form: accumulating it in FP32 between residual
// replacements injects rounding noise of relative size 2^-24 into every
// replaced residual, which the iteration then has to remove again.
//
// k_tstencil: each CTA owns 120 grid rows and walks a strip of L node
// columns. Column windows of every input are staged into shared memory by TMA
// bulk copies (cp.async.bulk) in groups of G columns, NG groups in flight,
// completion on one mbarrier per ring slot; one warp produces, one consumes.
// A consumer lane holds four consecutive rows (lanes 0..30 cover rows
// Y0-2 .. Y0+121), so the elements between its rows need no shuffle: per
// column only the node above its last row and the forces of the element below
// its first row cross lanes. Element arithmetic is issued on x/y pairs
// (packed FP32 instructions in the mixed form). Strips overlap by two
// columns; values there are recomputed from the inputs, never read from
// another strip's output, and the direction p ping-pongs between two buffers
// so no CTA overwrites what another still reads.
#pragma once

#include "common.cuh"
#include "layout.cuh"
#include "stencil.cuh"

namespace tpo {

constexpr int ST_THREADS = WPC * 32;  // 128 (k_blockpre)
// Stencil CTA: one consumer warp whose lanes hold LR consecutive grid rows
// each (lanes 0..30 cover rows Y0-2 .. Y0+121, the staged node window; lane 31
// mirrors lane 30 and its results are discarded), and one producer warp.
constexpr int LR = 4;
constexpr int TS_LANES = 31;
constexpr int TS_THREADS = 64;
static_assert(LR * TS_LANES == N_WIN, "the consumer lanes cover the staged node window");

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

// LR consecutive nodal pairs of a staged column from window index i0
// (a multiple of LR: 16-byte aligned for both storage types)
template <typename T>
__device__ __forceinline__ void lds_pairs(const V2<T> *col, int i0, V2<T> (&v)[LR]) {
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4 *>(col + i0);
    const float4 b = *reinterpret_cast<const float4 *>(col + i0 + 2);
    v[0] = make_float2(a.x, a.y);
    v[1] = make_float2(a.z, a.w);
    v[2] = make_float2(b.x, b.y);
    v[3] = make_float2(b.z, b.w);
  } else {
#pragma unroll
    for (int j = 0; j < LR; ++j) v[j] = col[i0 + j];
  }
}

// Element scales of a staged column at rows yb-1 .. yb+LR-1, e0 = the window
// index of row yb. The float window holds row yb-1 for every lane; in the
// double window lane 0's row yb-1 (= Y0-3) is not staged: it is only used for
// the preconditioner of row Y0-2, which is no output row, so the index is
// clamped to stay inside the window.
template <typename T>
__device__ __forceinline__ void lds_scales(const T *col, int e0, T (&s)[LR + 1]) {
  if constexpr (sizeof(T) == 4) {  // e0 = 2 (mod 4)
    s[0] = col[e0 - 1];
    const float2 a = *reinterpret_cast<const float2 *>(col + e0);
    const float2 b = *reinterpret_cast<const float2 *>(col + e0 + 2);
    s[1] = a.x;
    s[2] = a.y;
    s[3] = b.x;
    s[4] = b.y;
  } else {  // e0 = 0 (mod 4)
    s[0] = col[e0 > 0 ? e0 - 1 : 0];
    const double2 a = *reinterpret_cast<const double2 *>(col + e0);
    const double2 b = *reinterpret_cast<const double2 *>(col + e0 + 2);
    s[1] = a.x;
    s[2] = a.y;
    s[3] = b.x;
    s[4] = b.y;
  }
}

// the four fixed-mask bytes of rows yb .. yb+3 (byte j = row yb+j), i0 = 2 (mod 4)
__device__ __forceinline__ unsigned lds_mask4(const uint8_t *col, int i0) {
  const unsigned lo = *reinterpret_cast<const uint16_t *>(col + i0);
  const unsigned hi = *reinterpret_cast<const uint16_t *>(col + i0 + 2);
  return lo | (hi << 16);
}

// Store the pairs of rows j with bit j of `own` set, from slot0 (a multiple of
// two slots: 16-byte aligned for FP32 pairs). Whole 16-byte runs go out as one
// vector store.
template <typename T>
__device__ __forceinline__ void stg_pairs(T *base, size_t slot0, const V2<T> (&v)[LR],
                                          unsigned own) {
  V2<T> *p = reinterpret_cast<V2<T> *>(base) + slot0;
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int h = 0; h < LR; h += 2) {
      const unsigned two = (own >> h) & 3u;
      if (two == 3u)
        *reinterpret_cast<float4 *>(p + h) = make_float4(v[h].x, v[h].y, v[h + 1].x, v[h + 1].y);
      else if (two == 1u)
        p[h] = v[h];
      else if (two == 2u)
        p[h + 1] = v[h + 1];
    }
  } else {
#pragma unroll
    for (int j = 0; j < LR; ++j)
      if ((own >> j) & 1u) p[j] = v[j];
  }
}

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
  // the direction kernel reads z = M r as stored by the update kernel (or
  // the element-block preconditioner); it never rebuilds a preconditioner
  static_assert(MODE != M_DIR || PRE == TPO_PRECOND_BLOCK_JACOBI, "DIR reads the stored z");
  const int nx = a.nx, ny = a.ny, P = a.P;
  const int Y0 = bx * RPC;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int x0 = by * L;
  const int x1 = min(x0 + L, nx + 1);
  const int cA = x0 - 1;       // first staged column
  const int NC = x1 - cA + 1;  // staged columns cA..x1
  const int NGRP = (NC + G - 1) / G;
  const int ms = (Y0 + LEAD - 1) & ~15;  // first staged mask byte of a column

  const T *gs = static_cast<const T *>(a.s);
  const T *ga = static_cast<const T *>(a.a);
  T *src_p = nullptr, *dst_p = nullptr;
  if constexpr (MODE == M_DIR) {
    src_p = static_cast<T *>(parity ? a.pb : a.pa);
    dst_p = static_cast<T *>(parity ? a.pa : a.pb);
  }

  // ---- producer: stage group g into ring slot g % NG. A slot is reused only
  // after the consumer warp has released the group it held (empty[]).
  auto issue = [&](int g) {
    unsigned char *sb = smem + (g % NG) * SLOT;
    unsigned bytes = 0;
    for (int k = 0; k < G; ++k) {
      const int c = cA + g * G + k;
      if (c > x1) break;
      if (c >= 0 && c <= nx) bytes += Geo::CNB * (Geo::HAS_B ? 2 : 1) + Geo::CMB;
      if (c >= 0 && c < nx) bytes += Geo::CEB;
    }
    mbar_arrive_expect_tx(&full[g % NG], bytes);
    for (int k = 0; k < G; ++k) {
      const int c = cA + g * G + k;
      if (c > x1) break;
      if (c >= 0 && c <= nx) {
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
      mbar_init(&empty[s], 1);
    }
    fence_mbar_init();
  }
  __syncthreads();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;

  if (wid == 1) {
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
      if (!ok)  // let the copies this CTA started land before it exits
        for (int g = (issued > NG ? issued - NG : 0); g < issued; ++g)
          mbar_wait_bounded(&full[g % NG], (g / NG) & 1, nullptr, 0);
    }
  } else {

  // Lane l holds rows yb + j, j = 0..LR-1, yb = Y0 - 2 + LR l: node window
  // index LR l + j, element window index LR l + j + EOFF (EOFF = rows of the
  // element window below row Y0 - 2), mask byte m0 + j. Lane 31 reads lane
  // 30's rows (its results are discarded). Rows Y0 .. Y0 + RPC - 1 (and
  // <= ny) are this CTA's output rows.
  const int lq = min(lane, TS_LANES - 1);
  const int yb = Y0 - 2 + LR * lane;
  const int n0 = LR * lq;
  constexpr int EOFF = LEAD - 2 - EWin<T>::OFF;  // float: 2, double: 0
  const int e0 = n0 + EOFF;                       // element row yb (row yb - 1 is e0 - 1)
  const int m0 = Y0 + LEAD - 2 + n0 - ms;         // 2 (mod 4): u16-aligned
  unsigned own = 0;  // bit j: row yb + j is an output row of this CTA
#pragma unroll
  for (int j = 0; j < LR; ++j) {
    const int yj = yb + j;
    if (lane < TS_LANES && yj >= Y0 && yj < Y0 + RPC && yj <= ny) own |= 1u << j;
  }

  // Element-centric march along x. At step c the lane transforms its nodes
  // (c, yb+j) (p_new, or u with fixed DOFs zeroed), forms elements
  // (c-1, yb+j) from their corners (c-1, y) (c, y) (c, y+1) (c-1, y+1), and
  // finishes nodes (c-1, yb+j): carry[j] holds what elements (c-2, y) and
  // (c-2, y-1) gave node (c-1, y) one step earlier. The node above the lane's
  // last row comes from the next lane, the forces of the element below its
  // first row from the previous lane (two shuffles of pairs per column).
  const V2<C> zero2 = mk2<C>(C(0), C(0));
  V2<C> vp[LR + 1], carry[LR];
  C sp[LR + 1], sq[LR + 1];  // element columns c-1 and c-2, rows yb-1 .. yb+LR-1
  unsigned mp = 0;           // fixed-mask bytes of node column c-1 (byte j: row yb+j)
#pragma unroll
  for (int j = 0; j <= LR; ++j) {
    vp[j] = zero2;
    sp[j] = sq[j] = C(0);
    if (j < LR) carry[j] = zero2;
  }

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
    const bool node_ok = c >= 0 && c <= nx;
    const bool elem_ok = c >= 0 && c < nx;

    // ---- element scales of column c, rows yb-1 .. yb+LR-1
    C sc[LR + 1];
    if (elem_ok) {
      T sv[LR + 1];
      lds_scales<T>(colS, e0, sv);
#pragma unroll
      for (int j = 0; j <= LR; ++j) sc[j] = C(sv[j]);
    } else {
#pragma unroll
      for (int j = 0; j <= LR; ++j) sc[j] = C(0);
    }

    // ---- transformed nodal values at (c, yb+j)
    V2<C> v[LR + 1];
    unsigned mc = 0;
    if (node_ok) {
      mc = lds_mask4(colM, m0);
      V2<T> av[LR];
      lds_pairs<T>(colA, n0, av);
      if constexpr (MODE == M_DIR) {
        if (first) {
#pragma unroll
          for (int j = 0; j < LR; ++j) v[j] = cvt2<C, T>(av[j]);
        } else {
          V2<T> po[LR];
          lds_pairs<T>(colB, n0, po);
#pragma unroll
          for (int j = 0; j < LR; ++j)
            v[j] = fma2(bc2<C>(beta), cvt2<C, T>(po[j]), cvt2<C, T>(av[j]));
        }
#pragma unroll
        for (int j = 0; j < LR; ++j)  // the stored direction is what K sees
          v[j] = cvt2<C, T>(mk2<T>(T(v[j].x), T(v[j].y)));
      } else {
#pragma unroll
        for (int j = 0; j < LR; ++j) v[j] = cvt2<C, T>(av[j]);
        if constexpr (MODE == M_RES || MODE == M_RESX) {
          // u with fixed DOFs zeroed (idempotent write-back on owned nodes)
#pragma unroll
          for (int j = 0; j < LR; ++j) {
            const unsigned m = (mc >> (8 * j)) & 0xffu;
            if (m & FIXED_X) v[j].x = C(0);
            if (m & FIXED_Y) v[j].y = C(0);
            if (m && ((own >> j) & 1u) && c >= x0 && c < x1)
              st2<T>(static_cast<T *>(a.uw), pslot(c, yb + j, P), mk2<T>(T(v[j].x), T(v[j].y)));
          }
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < LR; ++j) v[j] = zero2;
    }
    v[LR] = shfl_down2<C>(v[0]);  // node (c, yb+LR)

    // ---- elements (c-1, yb+j): corners (c-1,y) (c,y) (c,y+1) (c-1,y+1)
    V2<C> fbl[LR], fbr[LR], ftr[LR], ftl[LR];
#pragma unroll
    for (int j = 0; j < LR; ++j)
      elem_forces2<C>(sp[j + 1], vp[j], v[j], v[j + 1], vp[j + 1], fbl[j], fbr[j], ftr[j], ftl[j]);
    const V2<C> tl_below = shfl_up2<C>(ftl[LR - 1]);  // element (c-1, yb-1) -> node (c-1, yb)
    const V2<C> tr_below = shfl_up2<C>(ftr[LR - 1]);  // element (c-1, yb-1) -> node (c, yb)

    // the consumer is done with group g: release its slot to the producer
    if (kk == G - 1 || k == NC - 1) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[g % NG]);
    }

    // ---- nodes (xo, yb+j), xo = c - 1, are complete
    const int xo = c - 1;
    if (own && xo >= x0) {
      const size_t node0 = pslot(xo, yb, P);
      V2<C> kv[LR];
#pragma unroll
      for (int j = 0; j < LR; ++j) {
        kv[j] = add2(add2(carry[j], fbl[j]), j ? ftl[j - 1] : tl_below);
        const unsigned m = (mp >> (8 * j)) & 0xffu;
        if (m & FIXED_X) kv[j].x = vp[j].x;  // identity rows at fixed DOFs
        if (m & FIXED_Y) kv[j].y = vp[j].y;
      }
      if constexpr (MODE == M_RAW || MODE == M_DIR) {
        V2<T> ks[LR];
#pragma unroll
        for (int j = 0; j < LR; ++j) {
          ks[j] = mk2<T>(T(kv[j].x), T(kv[j].y));
          if ((own >> j) & 1u) acc[0] += dot2d(vp[j], ks[j]);
        }
        if constexpr (MODE == M_DIR) {
          V2<T> pt[LR];
#pragma unroll
          for (int j = 0; j < LR; ++j) pt[j] = mk2<T>(T(vp[j].x), T(vp[j].y));
          stg_pairs<T>(dst_p, node0, pt, own);
        }
        stg_pairs<T>(static_cast<T *>(a.out), node0, ks, own);
      } else if constexpr (MODE == M_RES) {
        V2<T> rs[LR];
#pragma unroll
        for (int j = 0; j < LR; ++j) {
          rs[j] = mk2<T>(T(0), T(0));
          if (!((own >> j) & 1u)) continue;
          const V2<C> f = cvt2<C, T>(ld2<T>(static_cast<const T *>(a.f), node0 + j));
          rs[j] = mk2<T>(T(f.x - kv[j].x), T(f.y - kv[j].y));
          if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
            C pa, pb, pd;
            node_pre<C, PRE>((mp >> (8 * j)) & 0xffu, sq[j], sq[j + 1], sp[j], sp[j + 1], pa, pb,
                             pd);
            acc[0] += dot2d(rs[j], pre_apply<C>(pa, pb, pd, cvt2<C, T>(rs[j])));
          }
          acc[1] += dot2d(rs[j], rs[j]);
        }
        stg_pairs<T>(static_cast<T *>(a.out), node0, rs, own);
      } else {  // M_RESX: T == C == double; the inner solve stores FP32 and runs in FP32
        float2 r32[LR];
#pragma unroll
        for (int j = 0; j < LR; ++j) {
          r32[j] = make_float2(0.f, 0.f);
          if (!((own >> j) & 1u)) continue;
          const double2 f = ld2<double>(static_cast<const double *>(a.f), node0 + j);
          const double rx = f.x - (double)kv[j].x, ry = f.y - (double)kv[j].y;
          acc[0] += rx * rx + ry * ry;
          r32[j] = make_float2((float)rx, (float)ry);
          if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
            // the inner z = M r, formed as the inner kernels form it (FP32
            // scales and arithmetic)
            float pa, pb, pd;
            node_pre<float, PRE>((mp >> (8 * j)) & 0xffu, (float)sq[j], (float)sq[j + 1],
                                 (float)sp[j], (float)sp[j + 1], pa, pb, pd);
            acc[1] += dot2d(r32[j], pre_apply<float>(pa, pb, pd, r32[j]));
          }
          acc[2] += dot2d(r32[j], r32[j]);
        }
        stg_pairs<float>(static_cast<float *>(a.out), node0, r32, own);
      }
    }
#pragma unroll
    for (int j = 0; j < LR; ++j) carry[j] = add2(fbr[j], j ? ftr[j - 1] : tr_below);
#pragma unroll
    for (int j = 0; j <= LR; ++j) {
      vp[j] = v[j];
      sq[j] = sp[j];
      sp[j] = sc[j];
    }
    mp = mc;
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
// A thread takes UQ = 4 consecutive rows of one node column per pass, so
// every vector arrives as 16-byte loads (two per FP32 run of four nodes,
// four per FP64 run) and a thread has about 200 bytes in flight; no column
// walk. The node's four element scales come straight from the padded scale
// array: element (c-1, y-1), (c-1, y), (c, y-1), (c, y) sit at the node's
// slot - P - 1, - P, - 1 and + 0 (zero pads outside the grid rows). Only grid
// rows are written and summed.
constexpr int UF_THREADS = 256;
constexpr int UQ = 4;
static_assert(UQ == LR, "the run stores reuse stg_pairs");

// n / d for 0 <= n < 2^31 through a double reciprocal, corrected to exact
__device__ __forceinline__ int div_exact(int n, int d, double inv_d) {
  int q = (int)((double)n * inv_d);
  if ((q + 1) * d <= n) ++q;
  if (q * d > n) --q;
  return q;
}

// the nodal pairs of slots s0 .. s0+3 (s0 a multiple of 4: 32-byte aligned)
template <typename T>
__device__ __forceinline__ void ldg_quad(const T *__restrict__ base, size_t s0, V2<T> (&v)[UQ]) {
  if constexpr (sizeof(T) == 4) {
    const float4 *q = reinterpret_cast<const float4 *>(base + 2 * s0);
    const float4 a = q[0], b = q[1];
    v[0] = make_float2(a.x, a.y);
    v[1] = make_float2(a.z, a.w);
    v[2] = make_float2(b.x, b.y);
    v[3] = make_float2(b.z, b.w);
  } else {
    const double2 *q = reinterpret_cast<const double2 *>(base) + s0;
#pragma unroll
    for (int j = 0; j < UQ; ++j) v[j] = q[j];
  }
}

// scales of element column c at rows y0-1 .. y0+3 (e0 = the slot of row y0,
// a multiple of 4), zero for columns outside the grid or when not needed
template <typename T, typename C, bool NEED>
__device__ __forceinline__ void ldg_scales5(const T *__restrict__ s, int c, int nx, size_t e0,
                                            C (&o)[UQ + 1]) {
  if (!NEED || c < 0 || c >= nx) {
#pragma unroll
    for (int j = 0; j <= UQ; ++j) o[j] = C(0);
    return;
  }
  o[0] = C(s[e0 - 1]);
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4 *>(s + e0);
    o[1] = a.x;
    o[2] = a.y;
    o[3] = a.z;
    o[4] = a.w;
  } else {
    const double2 a = *reinterpret_cast<const double2 *>(s + e0);
    const double2 b = *reinterpret_cast<const double2 *>(s + e0 + 2);
    o[1] = C(a.x);
    o[2] = C(a.y);
    o[3] = C(b.x);
    o[4] = C(b.y);
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
  const int nx = a.nx, ny = a.ny, P = a.P;
  const int Q = (ny + 1 + UQ - 1) / UQ;  // runs of UQ rows per node column
  const double invQ = 1.0 / Q;
  const T *__restrict__ s = static_cast<const T *>(a.s);
  X *__restrict__ u = static_cast<X *>(a.u);
  T *__restrict__ r = static_cast<T *>(a.r);
  T *__restrict__ zo = static_cast<T *>(a.z);
  const T *__restrict__ ap = static_cast<const T *>(a.ap);
  const uint8_t *__restrict__ mask = a.mask;
  const int total = (nx + 1) * Q;
  double acc[2] = {0.0, 0.0};
  for (int n = bx * blockDim.x + threadIdx.x; n < total; n += gx * blockDim.x) {
    const int c = div_exact(n, Q, invQ), y0 = UQ * (n - c * Q);
    const size_t s0 = (size_t)c * P + LEAD + y0;
    unsigned ok = 0;  // bit j: row y0 + j is a grid row
#pragma unroll
    for (int j = 0; j < UQ; ++j)
      if (y0 + j <= ny) ok |= 1u << j;
    V2<X> uu[UQ];
    V2<T> rr[UQ], pp[UQ], aa[UQ];
    ldg_quad<X>(u, s0, uu);
    ldg_quad<T>(r, s0, rr);
    ldg_quad<T>(p, s0, pp);
    ldg_quad<T>(ap, s0, aa);
    C sl[UQ + 1], sr[UQ + 1];  // element columns c-1 and c, rows y0-1 .. y0+3
    ldg_scales5<T, C, PRE != TPO_PRECOND_NONE>(s, c - 1, nx, s0 - P, sl);
    ldg_scales5<T, C, PRE != TPO_PRECOND_NONE>(s, c, nx, s0, sr);
    const unsigned mq = *reinterpret_cast<const unsigned *>(mask + s0);
    V2<X> un[UQ];
    V2<T> rn[UQ], zt[UQ];
#pragma unroll
    for (int j = 0; j < UQ; ++j) {
      // the solution accumulates in FP64 in every form
      un[j] = mk2<X>(X(fma(alpha, (double)pp[j].x, (double)uu[j].x)),
                     X(fma(alpha, (double)pp[j].y, (double)uu[j].y)));
      rn[j] = mk2<T>(T(fmaT(-alpha_c, C(aa[j].x), C(rr[j].x))),
                     T(fmaT(-alpha_c, C(aa[j].y), C(rr[j].y))));
      C pa, pb, pd;
      node_pre<C, PRE>((mq >> (8 * j)) & 0xffu, sl[j], sl[j + 1], sr[j], sr[j + 1], pa, pb, pd);
      const V2<C> z = pre_apply<C>(pa, pb, pd, cvt2<C, T>(rn[j]));
      zt[j] = mk2<T>(T(z.x), T(z.y));
      if ((ok >> j) & 1u) {
        // r.z with the stored (rounded) z, the one the direction update uses
        acc[0] += zo ? dot2d(rn[j], zt[j]) : dot2d(rn[j], z);
        acc[1] += dot2d(rn[j], rn[j]);
      }
    }
    stg_pairs<X>(u, s0, un, ok);
    stg_pairs<T>(r, s0, rn, ok);
    if (zo) stg_pairs<T>(zo, s0, zt, ok);
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
  const int Q = (ny + 1 + UQ - 1) / UQ;
  const double invQ = 1.0 / Q;
  const int total = (nx + 1) * Q;
  for (int n = bx * blockDim.x + threadIdx.x; n < total; n += gx * blockDim.x) {
    const int c = div_exact(n, Q, invQ), y0 = UQ * (n - c * Q);
    const size_t s0 = (size_t)c * P + LEAD + y0;
    unsigned ok = 0;
#pragma unroll
    for (int j = 0; j < UQ; ++j)
      if (y0 + j <= ny) ok |= 1u << j;
    V2<T> rr[UQ], zt[UQ];
    ldg_quad<T>(r, s0, rr);
    C sl[UQ + 1], sr[UQ + 1];
    ldg_scales5<T, C, PRE != TPO_PRECOND_NONE>(s, c - 1, nx, s0 - P, sl);
    ldg_scales5<T, C, PRE != TPO_PRECOND_NONE>(s, c, nx, s0, sr);
    const unsigned mq = *reinterpret_cast<const unsigned *>(mask + s0);
#pragma unroll
    for (int j = 0; j < UQ; ++j) {
      C pa, pb, pd;
      node_pre<C, PRE>((mq >> (8 * j)) & 0xffu, sl[j], sl[j + 1], sr[j], sr[j + 1], pa, pb, pd);
      const V2<C> zz = pre_apply<C>(pa, pb, pd, cvt2<C, T>(rr[j]));
      zt[j] = mk2<T>(T(zz.x), T(zz.y));
    }
    stg_pairs<T>(z, s0, zt, ok);
  }
}
template <typename T, typename C, int PRE>
__global__ void __launch_bounds__(UF_THREADS) k_precond_flat(int nx, int ny, int P, const T *s,
                                                             const uint8_t *mask, const T *r,
                                                             T *z) {
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
};

template <typename T, typename C, bool INIT, int L, typename X = T>
__global__ void __launch_bounds__(ST_THREADS) k_blockpre(BlkArgs a) {
  PcgCtl *ctl = a.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
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
