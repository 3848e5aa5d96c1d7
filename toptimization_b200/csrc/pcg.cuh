// PCG kernels. One CG iteration is two launches:
//   k_stencil<DIR>   p = z + beta p (z from r on the fly, or the stored z of
//                    the element-block preconditioner), Ap = K p, p.Ap;
//                    its last CTA sets alpha (or flags a breakdown).
//   k_update / k_blockpre<UPDATE>
//                    u += alpha p, r -= alpha Ap, z = M r, r.z, ||r||^2;
//                    its last CTA tests convergence and sets beta.
// alpha, beta and the stop test never leave the device (PcgCtl). Every CTA
// reads the status word first and returns at once when the solve is over, so
// a host may enqueue more iterations than needed.
//
// Stencil kernels march along x: lane = grid row y, each thread walks a strip
// of L node columns keeping a 3x3 window of nodal values in registers; the
// y-neighbours come from warp shuffles. A warp computes 30 rows and uses its
// first and last lane only as halo (warps overlap by two rows), so every lane
// runs the same code. Strips overlap by one column on each side; values read
// there are recomputed from their inputs, never read back from a neighbouring
// strip's output, and the direction p ping-pongs between two buffers so that
// no CTA overwrites what another still reads.
#pragma once

#include "common.cuh"
#include "stencil.cuh"

namespace tpo {

constexpr int ST_THREADS = 128;  // 4 warps per CTA for the stencil kernels
constexpr int ROWS_PER_WARP = 30;

enum StMode { M_RAW = 0, M_DIR = 1, M_RES = 2, M_RESX = 3 };

struct StArgs {
  int nx, ny;
  const void *s;          // element scales (T)
  const uint8_t *fixed;   // per-node mask
  const void *in;         // RAW: x; RES/RESX: u
  void *out;              // RAW: y; DIR: Ap; RES: r; RESX: inner r (float)
  void *uw;               // RES/RESX: u written back with fixed DOFs zeroed
  const void *f;          // RES/RESX: right-hand side (T / double)
  const void *r;          // DIR: residual (point preconditioners)
  const void *z;          // DIR: stored z (element-block preconditioner)
  void *pa, *pb;          // DIR: direction buffers, src/dst chosen by it parity
  void *d;                // RESX: inner correction, zeroed
  double *part;           // partial sums
  PcgCtl *ctl;            // solve state (RESX: the inner solve)
  OuterCtl *octl;         // RESX: refinement state
  double *result;         // RAW: optional p.Ap output
};

// ---------------------------------------------------------------------------
// Stencil kernel: K applied to a transformed nodal field.
// ---------------------------------------------------------------------------
template <typename T, int MODE, int PRE, int L>
__global__ void __launch_bounds__(ST_THREADS) k_stencil(StArgs a) {
  constexpr int NV = (MODE == M_RAW || MODE == M_DIR) ? 1 : (MODE == M_RES ? 2 : 3);
  PcgCtl *ctl = a.ctl;
  double beta = 0.0;
  bool first = true;
  int parity = 0;
  if constexpr (MODE == M_DIR) {
    if (ctl->status != TPO_SOLVE_RUNNING) return;
    beta = ctl->beta;
    first = ctl->first != 0;
    parity = ctl->it & 1;
  }
  if constexpr (MODE == M_RESX) {
    if (a.octl->status != TPO_SOLVE_RUNNING) return;
  }
  const int nx = a.nx, ny = a.ny;
  const size_t ny1 = (size_t)ny + 1;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int y = gw * ROWS_PER_WARP - 1 + lane;
  const bool row_ok = (y >= 0) && (y <= ny);
  const bool own_row = row_ok && lane >= 1 && lane <= ROWS_PER_WARP;
  const int x0 = blockIdx.y * L;
  const int x1 = min(x0 + L, nx + 1);
  const T *__restrict__ s = static_cast<const T *>(a.s);

  const T *src_p = nullptr;
  T *dst_p = nullptr;
  if constexpr (MODE == M_DIR) {
    src_p = static_cast<const T *>(parity ? a.pb : a.pa);
    dst_p = static_cast<T *>(parity ? a.pa : a.pb);
  }

  // element scale columns c-2, c-1, c  (rows y-1 = d, y = u)
  T e0d = T(0), e0u = T(0), e1d = T(0), e1u = T(0), e2d, e2u;
  load_elem_col<T>(s, x0 - 2, y, nx, ny, e2d, e2u);
  // node columns c-2, c-1, c: values at rows y-1, y, y+1 and the mask at y
  const V2<T> zero2 = mk2<T>(T(0), T(0));
  V2<T> n0d = zero2, n0m = zero2, n0u = zero2, n1d = zero2, n1m = zero2, n1u = zero2;
  V2<T> n2d = zero2, n2m = zero2, n2u = zero2;
  unsigned m1 = 0, m2 = 0;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;

  // Raw inputs of one column, fetched one column ahead so that its loads are
  // in flight while the current column is computed.
  struct Raw {
    T sd, su;
    V2<T> a, b;
    unsigned m;
  };
  auto fetch = [&](int c, Raw &R) {
    load_elem_col<T>(s, c, y, nx, ny, R.sd, R.su);
    R.m = 0;
    R.a = zero2;
    R.b = zero2;
    if (row_ok && c >= 0 && c <= nx) {
      const size_t node = (size_t)c * ny1 + y;
      R.m = a.fixed[node];
      if constexpr (MODE == M_DIR) {
        if constexpr (PRE == TPO_PRECOND_BLOCK_JACOBI) R.a = ld2<T>(static_cast<const T *>(a.z), node);
        else R.a = ld2<T>(static_cast<const T *>(a.r), node);
        if (!first) R.b = ld2<T>(src_p, node);
      } else {
        R.a = ld2<T>(static_cast<const T *>(a.in), node);
      }
    }
  };
  Raw nxt;
  fetch(x0 - 1, nxt);

  for (int c = x0 - 1; c <= x1; ++c) {
    const Raw cur = nxt;
    if (c < x1) fetch(c + 1, nxt);
    e0d = e1d; e0u = e1u; e1d = e2d; e1u = e2u;
    e2d = cur.sd;
    e2u = cur.su;

    // ---- transformed nodal value at (c, y)
    V2<T> v = zero2;
    const unsigned m = cur.m;
    if (row_ok && c >= 0 && c <= nx) {
      if constexpr (MODE == M_RAW) {
        v = cur.a;
      } else if constexpr (MODE == M_DIR) {
        V2<T> z;
        if constexpr (PRE == TPO_PRECOND_BLOCK_JACOBI) z = cur.a;
        else z = point_precond<T, PRE>(cur.a, m, e1d, e1u, e2d, e2u);
        if (first) v = z;
        else v = mk2<T>(fmaT(T(beta), cur.b.x, z.x), fmaT(T(beta), cur.b.y, z.y));
      } else {  // M_RES, M_RESX: u with fixed DOFs zeroed (idempotent write-back)
        v = cur.a;
        if (m & FIXED_X) v.x = T(0);
        if (m & FIXED_Y) v.y = T(0);
        if (m && own_row && c >= x0 && c < x1)
          st2<T>(static_cast<T *>(a.uw), (size_t)c * ny1 + y, v);
      }
    }
    n0d = n1d; n0m = n1m; n0u = n1u;
    n1d = n2d; n1m = n2m; n1u = n2u;
    m1 = m2;
    m2 = m;
    n2m = v;
    n2d = shfl_up2<T>(v);
    n2u = shfl_down2<T>(v);

    // ---- output at node (xo, y), xo = c - 1
    const int xo = c - 1;
    if (own_row && xo >= x0) {
      const size_t node = (size_t)xo * ny1 + y;
      V2<T> kv = node_apply<T, false>(n0d, n0m, n0u, n1d, n1m, n1u, n2d, n2m, n2u, e0d, e0u,
                                      e1d, e1u);
      if (m1 & FIXED_X) kv.x = n1m.x;  // identity rows at fixed DOFs
      if (m1 & FIXED_Y) kv.y = n1m.y;
      if constexpr (MODE == M_RAW) {
        st2<T>(static_cast<T *>(a.out), node, kv);
        acc[0] += (double)n1m.x * kv.x + (double)n1m.y * kv.y;
      } else if constexpr (MODE == M_DIR) {
        st2<T>(dst_p, node, n1m);
        st2<T>(static_cast<T *>(a.out), node, kv);
        acc[0] += (double)n1m.x * kv.x + (double)n1m.y * kv.y;
      } else if constexpr (MODE == M_RES) {
        const V2<T> f = ld2<T>(static_cast<const T *>(a.f), node);
        const V2<T> r = mk2<T>(f.x - kv.x, f.y - kv.y);
        st2<T>(static_cast<T *>(a.out), node, r);
        if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
          const V2<T> z = point_precond<T, PRE>(r, m1, e0d, e0u, e1d, e1u);
          acc[0] += (double)r.x * z.x + (double)r.y * z.y;
        }
        acc[1] += (double)r.x * r.x + (double)r.y * r.y;
      } else {  // M_RESX: T == double; inner solve in float
        const double2 f = ld2<double>(static_cast<const double *>(a.f), node);
        const double rx = f.x - (double)kv.x, ry = f.y - (double)kv.y;
        acc[0] += rx * rx + ry * ry;
        const float2 r32 = make_float2((float)rx, (float)ry);
        st2<float>(static_cast<float *>(a.out), node, r32);
        st2<float>(static_cast<float *>(a.d), node, make_float2(0.f, 0.f));
        if constexpr (PRE != TPO_PRECOND_BLOCK_JACOBI) {
          const float2 z = point_precond<float, PRE>(r32, m1, (float)e0d, (float)e0u,
                                                     (float)e1d, (float)e1u);
          acc[1] += (double)r32.x * z.x + (double)r32.y * z.y;
        }
        acc[2] += (double)r32.x * r32.x + (double)r32.y * r32.y;
      }
    }
  }

  uint32_t *counter = (MODE == M_RESX) ? &a.octl->counter : &ctl->counter;
  if (!grid_reduce<NV>(acc, a.part, counter)) return;
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
    OuterCtl *o = a.octl;
    o->rr = acc[0];
    o->it += 1;
    if (!finite(acc[0])) {
      o->status = TPO_SOLVE_NONFINITE;
    } else if (acc[0] < o->tol_sq) {
      o->status = TPO_SOLVE_CONVERGED;
    }
    // (re)initialise the inner solve on this residual
    ctl->it = 0;
    ctl->first = 1;
    ctl->rr = acc[2];
    if (PRE != TPO_PRECOND_BLOCK_JACOBI) {
      ctl->rz = acc[1];
      ctl->tol_sq = ctl->rel_tol2 * acc[2];
    }
    ctl->status = (o->status == TPO_SOLVE_RUNNING) ? TPO_SOLVE_RUNNING : TPO_SOLVE_CONVERGED;
  }
}

// ---------------------------------------------------------------------------
// Point-preconditioner update: u += alpha p, r -= alpha Ap, z = M r (z not
// stored: the next direction kernel recomputes it), r.z and ||r||^2.
// Pointwise, so a warp covers 32 rows with no halo.
// ---------------------------------------------------------------------------
struct UpdArgs {
  int nx, ny;
  const void *s;
  const uint8_t *fixed;
  void *u, *r;
  const void *ap;
  const void *pa, *pb;
  double *part;
  PcgCtl *ctl;
};

__device__ __forceinline__ void finish_update(PcgCtl *ctl, double rz_new, double rr) {
  // reference solver.py:119-155: convergence on the recursive residual
  // before the direction update; beta = rz_new / (rz_old + 1e-60)
  ctl->it += 1;
  ctl->rr = rr;
  if (!finite(rz_new) || !finite(rr)) {
    ctl->status = TPO_SOLVE_NONFINITE;
  } else if (rr < ctl->tol_sq) {
    ctl->status = TPO_SOLVE_CONVERGED;
  } else if (ctl->it >= ctl->max_iter) {
    ctl->status = TPO_SOLVE_MAX_ITER;
  } else {
    ctl->beta = rz_new / (ctl->rz + 1e-60);
    ctl->rz = rz_new;
  }
}

template <typename T, int PRE, int L>
__global__ void __launch_bounds__(ST_THREADS) k_update(UpdArgs a) {
  PcgCtl *ctl = a.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const T alpha = T(ctl->alpha);
  const T *__restrict__ p = static_cast<const T *>((ctl->it & 1) ? a.pa : a.pb);
  const int nx = a.nx, ny = a.ny;
  const size_t ny1 = (size_t)ny + 1;
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  const bool row_ok = y <= ny;
  const int x0 = blockIdx.y * L;
  const int x1 = min(x0 + L, nx + 1);
  const T *__restrict__ s = static_cast<const T *>(a.s);
  T *__restrict__ u = static_cast<T *>(a.u);
  T *__restrict__ r = static_cast<T *>(a.r);
  const T *__restrict__ ap = static_cast<const T *>(a.ap);

  // Columns are processed in batches of UB: all loads of a batch are issued
  // before any of its arithmetic, so UB columns of loads are in flight.
  constexpr int UB = 4;
  T ebd = T(0), ebu = T(0);
  if (PRE != TPO_PRECOND_NONE) load_elem_col<T>(s, x0 - 1, y, nx, ny, ebd, ebu);
  double acc[2] = {0.0, 0.0};
  for (int cb = x0; cb < x1; cb += UB) {
    V2<T> uv[UB], rv[UB], pv[UB], av[UB];
    T sd[UB], su[UB];
    unsigned m[UB];
#pragma unroll
    for (int k = 0; k < UB; ++k) {
      const int c = cb + k;
      sd[k] = su[k] = T(0);
      m[k] = 0;
      if (c < x1) {
        if (PRE != TPO_PRECOND_NONE) load_elem_col<T>(s, c, y, nx, ny, sd[k], su[k]);
        if (row_ok) {
          const size_t node = (size_t)c * ny1 + y;
          m[k] = a.fixed[node];
          uv[k] = ld2<T>(u, node);
          rv[k] = ld2<T>(r, node);
          pv[k] = ld2<T>(p, node);
          av[k] = ld2<T>(ap, node);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < UB; ++k) {
      const int c = cb + k;
      const T ead = ebd, eau = ebu;
      ebd = sd[k];
      ebu = su[k];
      if (c < x1 && row_ok) {
        const size_t node = (size_t)c * ny1 + y;
        uv[k].x = fmaT(alpha, pv[k].x, uv[k].x);
        uv[k].y = fmaT(alpha, pv[k].y, uv[k].y);
        rv[k].x = fmaT(-alpha, av[k].x, rv[k].x);
        rv[k].y = fmaT(-alpha, av[k].y, rv[k].y);
        st2<T>(u, node, uv[k]);
        st2<T>(r, node, rv[k]);
        const V2<T> z = point_precond<T, PRE>(rv[k], m[k], ead, eau, ebd, ebu);
        acc[0] += (double)rv[k].x * z.x + (double)rv[k].y * z.y;
        acc[1] += (double)rv[k].x * rv[k].x + (double)rv[k].y * rv[k].y;
      }
    }
  }
  if (!grid_reduce<2>(acc, a.part, &ctl->counter)) return;
  if (threadIdx.x == 0) finish_update(ctl, acc[0], acc[1]);
}

// ---------------------------------------------------------------------------
// Element-block preconditioner (the reference's "block_jacobi",
// fem/preconditioner.py:47-108):
//   z = C^-1/2 sum_e w_e Ke_inv (C^-1/2 r)_e,  w_e = s_e / max(s_e, alpha)^2,
//   z[fixed] = 0,  C = elements per node.
// UPDATE: r_new = r - alpha Ap is formed for the strip and its halo (read from
// one residual buffer, written to the other), u += alpha p on owned nodes,
// then z from r_new, and the convergence/beta logic.
// INIT:   z from r as it is (first residual of a solve).
// ---------------------------------------------------------------------------
struct BlkArgs {
  int nx, ny;
  const void *w;        // element weights w_e (T)
  const uint8_t *fixed;
  void *u;
  const void *ap;
  const void *pa, *pb;  // directions (the one the current iteration wrote)
  void *ra, *rb;        // residual ping-pong
  void *z;
  double *part;
  PcgCtl *ctl;
};

template <typename T, bool INIT, int L>
__global__ void __launch_bounds__(ST_THREADS) k_blockpre(BlkArgs a) {
  PcgCtl *ctl = a.ctl;
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const int parity = ctl->it & 1;
  const T alpha = INIT ? T(0) : T(ctl->alpha);
  const T *r_src = static_cast<const T *>(INIT ? a.ra : (parity ? a.rb : a.ra));
  T *r_dst = static_cast<T *>(parity ? a.ra : a.rb);
  const T *__restrict__ p = static_cast<const T *>(parity ? a.pa : a.pb);
  const int nx = a.nx, ny = a.ny;
  const size_t ny1 = (size_t)ny + 1;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int y = gw * ROWS_PER_WARP - 1 + lane;
  const bool row_ok = (y >= 0) && (y <= ny);
  const bool own_row = row_ok && lane >= 1 && lane <= ROWS_PER_WARP;
  const int x0 = blockIdx.y * L;
  const int x1 = min(x0 + L, nx + 1);
  const T *__restrict__ w = static_cast<const T *>(a.w);
  T *__restrict__ u = static_cast<T *>(a.u);
  const T *__restrict__ ap = static_cast<const T *>(a.ap);
  T *__restrict__ z = static_cast<T *>(a.z);

  T e0d = T(0), e0u = T(0), e1d = T(0), e1u = T(0);
  const V2<T> zero2 = mk2<T>(T(0), T(0));
  V2<T> n0d = zero2, n0m = zero2, n0u = zero2, n1d = zero2, n1m = zero2, n1u = zero2;
  V2<T> n2d = zero2, n2m = zero2, n2u = zero2;
  V2<T> rn1 = zero2, rn2 = zero2;  // unscaled residual at columns c-1, c
  unsigned m1 = 0, m2 = 0;
  double acc[2] = {0.0, 0.0};

  // raw inputs of column c, fetched one column ahead
  struct Raw {
    T wd, wu;
    V2<T> r, ap, u, p;
    unsigned m;
  };
  auto fetch = [&](int c, Raw &R) {
    load_elem_col<T>(w, c - 1, y, nx, ny, R.wd, R.wu);
    R.m = 0;
    R.r = R.ap = R.u = R.p = zero2;
    if (row_ok && c >= 0 && c <= nx) {
      const size_t node = (size_t)c * ny1 + y;
      R.m = a.fixed[node];
      R.r = ld2<T>(r_src, node);
      if (!INIT) {
        R.ap = ld2<T>(ap, node);
        if (own_row && c >= x0 && c < x1) {
          R.u = ld2<T>(u, node);
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
    V2<T> rt = zero2, rn = zero2;
    const unsigned m = cur.m;
    if (row_ok && c >= 0 && c <= nx) {
      const size_t node = (size_t)c * ny1 + y;
      rn = cur.r;
      if (!INIT) {
        rn.x = fmaT(-alpha, cur.ap.x, rn.x);
        rn.y = fmaT(-alpha, cur.ap.y, rn.y);
        if (own_row && c >= x0 && c < x1) {
          V2<T> uv = cur.u;
          uv.x = fmaT(alpha, cur.p.x, uv.x);
          uv.y = fmaT(alpha, cur.p.y, uv.y);
          st2<T>(u, node, uv);
          st2<T>(r_dst, node, rn);
        }
      }
      const T sq = sqrt(T(node_elem_count(c, y, nx, ny)));
      rt = mk2<T>(rn.x / sq, rn.y / sq);
    }
    n0d = n1d; n0m = n1m; n0u = n1u;
    n1d = n2d; n1m = n2m; n1u = n2u;
    rn1 = rn2; rn2 = rn;
    m1 = m2; m2 = m;
    n2m = rt;
    n2d = shfl_up2<T>(rt);
    n2u = shfl_down2<T>(rt);

    const int xo = c - 1;
    if (own_row && xo >= x0) {
      const size_t node = (size_t)xo * ny1 + y;
      V2<T> zz = node_apply<T, true>(n0d, n0m, n0u, n1d, n1m, n1u, n2d, n2m, n2u, e0d, e0u, e1d,
                                     e1u);
      const T sq = sqrt(T(node_elem_count(xo, y, nx, ny)));
      zz.x = (m1 & FIXED_X) ? T(0) : zz.x / sq;
      zz.y = (m1 & FIXED_Y) ? T(0) : zz.y / sq;
      st2<T>(z, node, zz);
      acc[0] += (double)rn1.x * zz.x + (double)rn1.y * zz.y;
      acc[1] += (double)rn1.x * rn1.x + (double)rn1.y * rn1.y;
    }
  }
  if (!grid_reduce<2>(acc, a.part, &ctl->counter)) return;
  if (threadIdx.x != 0) return;
  if (INIT) {
    ctl->rz = acc[0];
    ctl->rr = acc[1];
    if (ctl->rel_tol2 > 0.0) ctl->tol_sq = ctl->rel_tol2 * acc[1];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  } else {
    finish_update(ctl, acc[0], acc[1]);
  }
}

// ---------------------------------------------------------------------------
// Per-solve setup and small helpers
// ---------------------------------------------------------------------------
// s = e_min + rho^p (1 - e_min) (reference fem/kernels.py:92), its FP32 copy,
// and the element-block weights w = s / max(s, alpha)^2 (preconditioner.py:55-57).
__global__ void k_scales(int n, const double *__restrict__ rho, double e_min, double pen,
                         double alpha_reg, double *__restrict__ s64, float *__restrict__ s32,
                         double *__restrict__ w64, float *__restrict__ w32) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const double s = e_min + pow(rho[e], pen) * (1.0 - e_min);
    if (s64) s64[e] = s;
    if (s32) s32[e] = (float)s;
    if (w64 || w32) {
      const double sc = fmax(s, alpha_reg);
      const double w = s / (sc * sc);
      if (w64) w64[e] = w;
      if (w32) w32[e] = (float)w;
    }
  }
}

template <typename T>
__global__ void k_scales_t(int n, const T *__restrict__ rho, double e_min, double pen,
                           T *__restrict__ s) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    s[e] = T(e_min + pow((double)rho[e], pen) * (1.0 - e_min));
  }
}

__global__ void k_ctl_init(PcgCtl *ctl, double tol_sq, double rel_tol2, int max_iter,
                           OuterCtl *octl, double outer_tol_sq) {
  ctl->rz = 0.0;
  ctl->alpha = 0.0;
  ctl->beta = 0.0;
  ctl->rr = 0.0;
  ctl->pap = 0.0;
  ctl->tol_sq = tol_sq;
  ctl->rel_tol2 = rel_tol2;
  ctl->it = 0;
  ctl->status = TPO_SOLVE_RUNNING;
  ctl->max_iter = max_iter;
  ctl->first = 1;
  ctl->counter = 0u;
  if (octl) {
    octl->rr = 0.0;
    octl->tol_sq = outer_tol_sq;
    octl->it = 0;
    octl->status = TPO_SOLVE_RUNNING;
    octl->counter = 0u;
  }
}

// Mixed precision: u += d (FP32 correction) on every DOF.
__global__ void k_correct(size_t n2, double *__restrict__ u, const float *__restrict__ d) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2;
       i += (size_t)gridDim.x * blockDim.x) {
    u[i] += (double)d[i];
  }
}

}  // namespace tpo
