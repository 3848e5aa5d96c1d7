// Node-centric Q4 stencil: the rows of K(rho) (or of the element-block
// preconditioner) that belong to one node, gathered from its four elements.
//
// The reference scatters each element's Ke p_e into the nodes with atomics
// (src/toptimization/fem/kernels.py:143-176). Here each node gathers the two
// rows of its four elements instead: no atomics, one write per DOF, and the
// four element contributions are added in ascending element index, the order
// a serial scatter would use.
//
// Element (ex, ey) has corners, local order 0..3: (ex,ey) (ex+1,ey)
// (ex+1,ey+1) (ex,ey+1). Node (x, y) is corner 2 of element (x-1,y-1),
// corner 1 of (x-1,y), corner 3 of (x,y-1) and corner 0 of (x,y).
#pragma once

#include "common.cuh"

namespace tpo {

// acc += s * K[2A:2A+2, :] . (q0, q1, q2, q3)   (K = Ke, or Ke_inv if INV)
template <int A, typename T, bool INV>
__device__ __forceinline__ void elem_rows(V2<T> &acc, T s, V2<T> q0, V2<T> q1, V2<T> q2,
                                          V2<T> q3) {
  const T q[8] = {q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y};
  T ax = kmat<T, INV>((2 * A) * 8) * q[0];
  T ay = kmat<T, INV>((2 * A + 1) * 8) * q[0];
#pragma unroll
  for (int j = 1; j < 8; ++j) {
    ax = fmaT(kmat<T, INV>((2 * A) * 8 + j), q[j], ax);
    ay = fmaT(kmat<T, INV>((2 * A + 1) * 8 + j), q[j], ay);
  }
  acc.x = fmaT(s, ax, acc.x);
  acc.y = fmaT(s, ay, acc.y);
}

// Rows of node (x, y) applied to the 3x3 neighbourhood of nodal values
// (L/C/R = columns x-1, x, x+1; D/M/U = rows y-1, y, y+1) with element
// scales s_ll = s(x-1,y-1), s_lh = s(x-1,y), s_rl = s(x,y-1), s_rh = s(x,y).
template <typename T, bool INV>
__device__ __forceinline__ V2<T> node_apply(V2<T> LD, V2<T> LM, V2<T> LU, V2<T> CD, V2<T> CM,
                                            V2<T> CU, V2<T> RD, V2<T> RM, V2<T> RU, T s_ll,
                                            T s_lh, T s_rl, T s_rh) {
  V2<T> acc = mk2<T>(T(0), T(0));
  elem_rows<2, T, INV>(acc, s_ll, LD, CD, CM, LM);  // element (x-1, y-1)
  elem_rows<1, T, INV>(acc, s_lh, LM, CM, CU, LU);  // element (x-1, y)
  elem_rows<3, T, INV>(acc, s_rl, CD, RD, RM, CM);  // element (x,   y-1)
  elem_rows<0, T, INV>(acc, s_rh, CM, RM, RU, CU);  // element (x,   y)
  return acc;
}

// s * Ke * p_e for one element from its corner values (BL, BR, TR, TL), using
// Ke = B0^T D B0 + ch (hx hx^T + hy hy^T): the centre strain (ex, ey, g) and
// the two hourglass amplitudes are formed once, then spread to the corners.
// About 40 flops instead of the 64 multiply-adds of the dense 8x8 product.
template <typename T>
__device__ __forceinline__ void elem_forces(T s, V2<T> bl, V2<T> br, V2<T> tr, V2<T> tl,
                                            V2<T> &fbl, V2<T> &fbr, V2<T> &ftr, V2<T> &ftl) {
  const T a = tr.x - bl.x, b = br.x - tl.x;    // x: diagonal differences
  const T ay = tr.y - bl.y, by = br.y - tl.y;  // y: diagonal differences
  const T apb = a + b, ayb = ay - by;
  const T P = s * fmaT(kst<T>(0), apb, kst<T>(1) * ayb);
  const T R = s * fmaT(kst<T>(1), apb, kst<T>(0) * ayb);
  const T Q = s * kst<T>(2) * ((a - b) + (ay + by));
  const T sh = s * kst<T>(3);
  const T hx = sh * ((bl.x + tr.x) - (br.x + tl.x));
  const T hy = sh * ((bl.y + tr.y) - (br.y + tl.y));
  const T PQ = P + Q, PmQ = P - Q, RQ = R + Q, RmQ = R - Q;
  fbl = mk2<T>(hx - PQ, hy - RQ);
  fbr = mk2<T>(PmQ - hx, -(RmQ + hy));
  ftr = mk2<T>(PQ + hx, RQ + hy);
  ftl = mk2<T>(-(PmQ + hx), RmQ - hy);
}

// Point preconditioners computed on the fly from the node's four element
// scales (same argument order as node_apply).
//  JACOBI: z = r / diag, diag_i = sum_e s_e Ke_ii, fixed -> 1, floor 1e-20
//          (reference fem/kernels.py:65-101).
//  NODAL:  z = B^-1 r, B = sum_e s_e Ke[2a:2a+2, 2a:2a+2], fixed DOFs get an
//          identity row and column (no reference counterpart).
//  NONE:   z = r.
template <typename T, int PRE>
__device__ __forceinline__ V2<T> point_precond(V2<T> r, unsigned m, T s_ll, T s_lh, T s_rl,
                                               T s_rh) {
  if constexpr (PRE == TPO_PRECOND_JACOBI) {
    // element order: (x-1,y-1) corner 2, (x-1,y) corner 1, (x,y-1) corner 3, (x,y) corner 0
    T dx = s_ll * kmat<T, false>(4 * 8 + 4);
    dx = fmaT(s_lh, kmat<T, false>(2 * 8 + 2), dx);
    dx = fmaT(s_rl, kmat<T, false>(6 * 8 + 6), dx);
    dx = fmaT(s_rh, kmat<T, false>(0 * 8 + 0), dx);
    T dy = s_ll * kmat<T, false>(5 * 8 + 5);
    dy = fmaT(s_lh, kmat<T, false>(3 * 8 + 3), dy);
    dy = fmaT(s_rl, kmat<T, false>(7 * 8 + 7), dy);
    dy = fmaT(s_rh, kmat<T, false>(1 * 8 + 1), dy);
    if (m & FIXED_X) dx = T(1); else if (dx < T(1e-20)) dx = T(1e-20);
    if (m & FIXED_Y) dy = T(1); else if (dy < T(1e-20)) dy = T(1e-20);
    return mk2<T>(r.x / dx, r.y / dy);
  } else if constexpr (PRE == TPO_PRECOND_NODAL_BLOCK) {
    T bxx = s_ll * kmat<T, false>(4 * 8 + 4);
    bxx = fmaT(s_lh, kmat<T, false>(2 * 8 + 2), bxx);
    bxx = fmaT(s_rl, kmat<T, false>(6 * 8 + 6), bxx);
    bxx = fmaT(s_rh, kmat<T, false>(0 * 8 + 0), bxx);
    T bxy = s_ll * kmat<T, false>(4 * 8 + 5);
    bxy = fmaT(s_lh, kmat<T, false>(2 * 8 + 3), bxy);
    bxy = fmaT(s_rl, kmat<T, false>(6 * 8 + 7), bxy);
    bxy = fmaT(s_rh, kmat<T, false>(0 * 8 + 1), bxy);
    T byy = s_ll * kmat<T, false>(5 * 8 + 5);
    byy = fmaT(s_lh, kmat<T, false>(3 * 8 + 3), byy);
    byy = fmaT(s_rl, kmat<T, false>(7 * 8 + 7), byy);
    byy = fmaT(s_rh, kmat<T, false>(1 * 8 + 1), byy);
    if (m & FIXED_X) { bxx = T(1); bxy = T(0); }
    if (m & FIXED_Y) { byy = T(1); bxy = T(0); }
    const T det = bxx * byy - bxy * bxy;
    if (det > T(0)) {
      const T inv = T(1) / det;
      return mk2<T>((byy * r.x - bxy * r.y) * inv, (bxx * r.y - bxy * r.x) * inv);
    }
    // degenerate block (only with e_min = 0 and void neighbourhoods): Jacobi
    return mk2<T>(r.x / fmax(bxx, T(1e-20)), r.y / fmax(byy, T(1e-20)));
  } else {
    return r;
  }
}

// 1/x for x inside FP32's normal range: the approximate FP32 reciprocal
// (rcp.approx, relative error below 2^-22) as the seed, then two Newton-Raphson
// steps y <- y + y (1 - x y) in FP64, each of which squares the relative error
// (2^-22 -> 2^-44 -> below FP64 rounding).
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rcp_nr(double x) {
  double y = (double)rcp_approx((float)x);
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
// reciprocal in the preconditioner's arithmetic type: FP64 as above, FP32 the
// correctly rounded single-precision reciprocal
__device__ __forceinline__ double rcpT(double x) { return rcp_nr(x); }
__device__ __forceinline__ float rcpT(float x) { return __frcp_rn(x); }

// z = [[a, b], [b, d]] r: the point preconditioner of node (x, y) from its
// four element scales (s_ll = (x-1,y-1), s_lh = (x-1,y), s_rl = (x,y-1),
// s_rh = (x,y)). Same operator as point_precond (stencil.cuh), written for
// the square-Q4 Ke: every diagonal entry is K00, and the x-y entry of
// corner a's block is +K01, -K01, +K01, -K01 for a = 0..3.
//  JACOBI: diag = K00 sum(s) (fixed DOF -> 1, floor 1e-20), reference
//          fem/kernels.py:65-101.
//  NODAL:  B = [[K00 S, K01 D], [K01 D, K00 S]], S = sum(s),
//          D = s_ll - s_lh - s_rl + s_rh (the corner signs), fixed DOFs get an
//          identity row and column; a singular block falls back to Jacobi.
template <typename C, int PRE>
__device__ __forceinline__ void node_pre(unsigned m, C s_ll, C s_lh, C s_rl, C s_rh, C &a, C &b,
                                         C &d) {
  if constexpr (PRE == TPO_PRECOND_NONE) {
    a = d = C(1);
    b = C(0);
  } else {
    const C k00 = kst<C>(4);
    const C S = (s_ll + s_lh) + (s_rl + s_rh);
    C bxx = k00 * S, byy = bxx;
    if constexpr (PRE == TPO_PRECOND_JACOBI) {
      if (m & FIXED_X) bxx = C(1); else if (bxx < C(1e-20)) bxx = C(1e-20);
      if (m & FIXED_Y) byy = C(1); else if (byy < C(1e-20)) byy = C(1e-20);
      a = rcpT(bxx);
      d = (byy == bxx) ? a : rcpT(byy);
      b = C(0);
    } else {
      C bxy = kst<C>(5) * ((s_ll - s_lh) + (s_rh - s_rl));
      if (m & FIXED_X) { bxx = C(1); bxy = C(0); }
      if (m & FIXED_Y) { byy = C(1); bxy = C(0); }
      const C det = bxx * byy - bxy * bxy;
      if (det > C(1e-36)) {
        const C inv = rcpT(det);
        a = byy * inv;
        d = bxx * inv;
        b = -bxy * inv;
      } else if (det > C(0)) {
        const C inv = C(1) / det;
        a = byy * inv;
        d = bxx * inv;
        b = -bxy * inv;
      } else {
        a = C(1) / fmax(bxx, C(1e-20));
        d = C(1) / fmax(byy, C(1e-20));
        b = C(0);
      }
    }
  }
}

template <typename C>
__device__ __forceinline__ V2<C> pre_apply(C a, C b, C d, V2<C> r) {
  return mk2<C>(fmaT(a, r.x, b * r.y), fmaT(b, r.x, d * r.y));
}

// Elements sharing node (x, y) -- the reference's diag_count
// (fem/preconditioner.py:19-30), here from the grid position.
__device__ __forceinline__ int node_elem_count(int x, int y, int nx, int ny) {
  const int cx = (x >= 1) + (x <= nx - 1);
  const int cy = (y >= 1) + (y <= ny - 1);
  return cx * cy;
}

// Scales of element column c at rows y-1 (sd) and y (su), zero outside the
// grid (the zero padding makes boundary nodes need no special case).
template <typename T>
__device__ __forceinline__ void load_elem_col(const T *__restrict__ s, int c, int y, int nx,
                                              int ny, T &sd, T &su) {
  sd = T(0);
  su = T(0);
  if (c >= 0 && c < nx) {
    const T *col = s + (size_t)c * ny;
    if (y >= 1 && y <= ny) sd = __ldg(col + (y - 1));
    if (y >= 0 && y < ny) su = __ldg(col + y);
  }
}

}  // namespace tpo
