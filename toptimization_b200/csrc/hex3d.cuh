// 3D path: trilinear hexahedra (H8) on a structured nelx x nely x nelz grid of
// unit cubes. Reference: fem/kernels.py:104-129 (diagonal), :179-212
// (matvec), :275-308 (sensitivity); fem/fused_kernels.py:59-94 (matvec + p.Ap);
// fem/preconditioner.py:34-44,112-156 (element-block preconditioner);
// optimizer/filter.py:75-97 (3D filter box).
//
// Layouts are the reference's numbering (mesh.py:68-112), used as they are:
//   node (ix, iy, iz)    -> (ix*(nely+1) + iy)*(nelz+1) + iz    (iz fastest)
//   nodal vector v       -> v[3*node + {0:x, 1:y, 2:z}]
//   element (ex, ey, ez) -> (ex*nely + ey)*nelz + ez
//   fixed mask           -> uint8 per node, bit0/1/2 = x/y/z fixed
//
// The stiffness applications (matvec, PCG direction, first residual) run
// element-centric with a structured H8 operator (k_hex_elem, below) when the
// stiffness has the isotropic unit-cube form, which tpo_set_stiffness3
// checks. The element-block preconditioner, and any other stiffness, use a
// gather: one thread per node sums the rows of its (up to) eight elements.
// Thread n reads the 27-node neighbourhood once (3 values each) and keeps one
// partial 3-vector per incident element,
//   y_k += Ke[3a+c][3b+j] v_m[j]      (a: the node's corner in element k,
//                                       b: neighbour m's corner),
// then scales each by its element weight: 64 node pairs x 9 multiply-adds +
// 24 = 600 FP64 FMAs per node, no atomics, a fixed summation order. All
// corner indices are compile-time constants after unrolling, so every Ke entry
// is a constant-bank operand. At these arithmetic intensities the FP64 pipe,
// not HBM, is the bound (576 FMAs against ~57 bytes per node).
#pragma once

#include "common.cuh"

namespace tpo {

// 24x24 H8 stiffness and its regularised inverse (element-block
// preconditioner), row-major, DOFs [x,y,z] per corner in mesh.py:87-96 order.
__constant__ double c_ke3[576];
__constant__ double c_kinv3[576];

constexpr int H3_THREADS = 128;  // gather kernels
constexpr int H3_FLAT = 256;     // pointwise kernels
constexpr int H3_MAXR = 8;       // filter: ceil(rmin) <= 8

struct Hex3 {
  int nx, ny, nz;  // elements per axis
  __host__ __device__ int64_t nodes() const { return (int64_t)(nx + 1) * (ny + 1) * (nz + 1); }
  __host__ __device__ int64_t elems() const { return (int64_t)nx * ny * nz; }
};

// H8 corner index of offset (dx, dy, dz) in {0,1}^3: bottom face (z = 0)
// counter-clockwise from (0,0), then the top face (reference mesh.py:87-96).
__host__ __device__ constexpr int h8_corner(int dx, int dy, int dz) {
  return 4 * dz + (dy ? (dx ? 2 : 3) : (dx ? 1 : 0));
}

template <bool INV> __device__ __forceinline__ double kent3(int i);
template <> __device__ __forceinline__ double kent3<false>(int i) { return c_ke3[i]; }
template <> __device__ __forceinline__ double kent3<true>(int i) { return c_kinv3[i]; }

struct NodePos {
  int ix, iy, iz;
  int64_t n;
};

__device__ __forceinline__ NodePos node_pos(const Hex3 &g, int64_t n) {
  NodePos p;
  p.n = n;
  const int64_t nz1 = g.nz + 1, ny1 = g.ny + 1;
  const int64_t col = n / nz1;
  p.iz = (int)(n - col * nz1);
  p.ix = (int)(col / ny1);
  p.iy = (int)(col - (int64_t)p.ix * ny1);
  return p;
}

// Element weights around a node: k = (ex*2 + ey)*2 + ez for the element with
// origin (ix-1+ex, iy-1+ey, iz-1+ez); 0 outside the grid.
__device__ __forceinline__ void node_elem_weights(const Hex3 &g, const NodePos &p,
                                                  const double *__restrict__ w, double (&we)[8]) {
#pragma unroll
  for (int ex = 0; ex < 2; ++ex)
#pragma unroll
    for (int ey = 0; ey < 2; ++ey)
#pragma unroll
      for (int ez = 0; ez < 2; ++ez) {
        const int x = p.ix - 1 + ex, y = p.iy - 1 + ey, z = p.iz - 1 + ez;
        const bool ok = x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz;
        we[(ex * 2 + ey) * 2 + ez] = ok ? w[((int64_t)x * g.ny + y) * g.nz + z] : 0.0;
      }
}

// 1/sqrt(number of elements at a node) (elements sharing each of its DOFs,
// reference preconditioner.py:34-44): the count is a product of three
// factors 1 or 2, so the root is one of four constants.
__device__ __forceinline__ double inv_sqrt_count(const Hex3 &g, int ix, int iy, int iz) {
  const int k = (ix > 0 && ix < g.nx) + (iy > 0 && iy < g.ny) + (iz > 0 && iz < g.nz);
  return k == 0 ? 1.0 : k == 1 ? 0.70710678118654752440 : k == 2 ? 0.5 : 0.35355339059327376220;
}

// out[c] = sum_k we[k] sum_{b,j} M[3a_k+c][3b+j] v(b)[j] over the node's 8
// elements; load(ox, oy, oz, v) returns neighbour (ix+ox, iy+oy, iz+oz)'s three
// values (zeros outside the grid).
template <bool INV, typename Load>
__device__ __forceinline__ void hex_gather(const double (&we)[8], Load load, double (&out)[3]) {
  double y[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k) y[k][0] = y[k][1] = y[k][2] = 0.0;
#pragma unroll
  for (int ox = -1; ox <= 1; ++ox)
#pragma unroll
    for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
      for (int oz = -1; oz <= 1; ++oz) {
        double v[3];
        load(ox, oy, oz, v);
#pragma unroll
        for (int ex = 0; ex < 2; ++ex)
#pragma unroll
          for (int ey = 0; ey < 2; ++ey)
#pragma unroll
            for (int ez = 0; ez < 2; ++ez) {
              const int bx = ox + 1 - ex, by = oy + 1 - ey, bz = oz + 1 - ez;
              if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
              const int a = h8_corner(1 - ex, 1 - ey, 1 - ez);
              const int b = h8_corner(bx, by, bz);
              const int k = (ex * 2 + ey) * 2 + ez;
#pragma unroll
              for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                  y[k][c] = fma(kent3<INV>((3 * a + c) * 24 + 3 * b + j), v[j], y[k][c]);
            }
      }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) t = fma(we[k], y[k][c], t);
    out[c] = t;
  }
}

// in-grid neighbour test and its flat node index
struct Nbr {
  const Hex3 &g;
  const NodePos &p;
  int64_t sx, sy;  // node strides along x, y
  __device__ __forceinline__ bool at(int ox, int oy, int oz, int64_t &m) const {
    const int x = p.ix + ox, y = p.iy + oy, z = p.iz + oz;
    m = p.n + ox * sx + oy * sy + oz;
    return x >= 0 && x <= g.nx && y >= 0 && y <= g.ny && z >= 0 && z <= g.nz;
  }
};

// ---------------------------------------------------------------------------
// Gather kernels
// ---------------------------------------------------------------------------
enum Hex3Mode {
  H3_APPLY = 0,  // ap = K p (fixed rows: p), p.ap
  H3_RES = 1,    // r = f - K u, z = r / diag (or r), r.z, ||r||^2: first residual
  H3_DIR = 2,    // p' = z + beta p (p' = z first), ap = K p', p'.ap -> alpha
  H3_BLOCK = 3   // z = element-block M r, r.z, ||r||^2 -> stop / beta
};

struct Hex3Args {
  Hex3 g;
  const double *w;       // element weights: SIMP scales (block: s / max(s, alpha)^2)
  const uint8_t *mask;
  const double *x;       // APPLY: p; RES: u; DIR: z; BLOCK: r
  double *pa, *pb;       // DIR: direction ping-pong pair (by the parity of ctl->it)
  const double *f;       // RES: load
  const double *diag;    // RES: Jacobi diagonal (nullptr: no preconditioner)
  double *out;           // APPLY/DIR: ap; RES: r; BLOCK: z
  double *z;             // RES: z (Jacobi)
  double *part;
  PcgCtl *ctl;           // RES/DIR/BLOCK
  uint32_t *counter;     // APPLY
  double *pap_out;       // APPLY (nullable)
  int init;              // BLOCK: first residual of the solve
};

template <int MODE, int PRE>
__global__ void __launch_bounds__(H3_THREADS) k_hex_gather(Hex3Args a) {
  PcgCtl *ctl = a.ctl;
  if (MODE != H3_APPLY && ctl->status != TPO_SOLVE_RUNNING) return;
  const Hex3 g = a.g;
  const int64_t total = g.nodes();
  const int64_t sy = g.nz + 1, sx = (int64_t)(g.ny + 1) * sy;
  bool first = true;
  double beta = 0.0;
  const double *pold = nullptr;
  double *pnew = nullptr;
  if (MODE == H3_DIR) {
    first = ctl->first != 0;
    beta = ctl->beta;
    // iteration k reads the direction of k-1 and writes its own into the other
    // buffer; the update kernel of iteration k reads it from there
    const bool odd = ctl->it & 1;
    pold = odd ? a.pb : a.pa;
    pnew = odd ? a.pa : a.pb;
  }
  double acc[2] = {0.0, 0.0};
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < total;
       n += (int64_t)gridDim.x * blockDim.x) {
    const NodePos p = node_pos(g, n);
    const Nbr nb{g, p, sx, sy};
    double we[8];
    node_elem_weights(g, p, a.w, we);
    double own[3] = {0.0, 0.0, 0.0};  // this node's input values (direction: p')
    double o[3];
    auto load = [&](int ox, int oy, int oz, double (&v)[3]) {
      int64_t m;
      const bool ok = nb.at(ox, oy, oz, m);
#pragma unroll
      for (int j = 0; j < 3; ++j) v[j] = 0.0;
      if (ok) {
        const double *src = a.x + 3 * m;
#pragma unroll
        for (int j = 0; j < 3; ++j) v[j] = src[j];
        if (MODE == H3_DIR && !first) {
          const double *po = pold + 3 * m;
#pragma unroll
          for (int j = 0; j < 3; ++j) v[j] = fma(beta, po[j], v[j]);
        }
        if (MODE == H3_BLOCK) {
          const double s = inv_sqrt_count(g, p.ix + ox, p.iy + oy, p.iz + oz);
#pragma unroll
          for (int j = 0; j < 3; ++j) v[j] *= s;
        }
      }
      if (ox == 0 && oy == 0 && oz == 0) {
#pragma unroll
        for (int j = 0; j < 3; ++j) own[j] = v[j];
      }
    };
    hex_gather<MODE == H3_BLOCK>(we, load, o);
    const unsigned fm = a.mask[n];
    double *dst = a.out + 3 * n;
    if (MODE == H3_APPLY || MODE == H3_DIR) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double ap = ((fm >> c) & 1u) ? own[c] : o[c];
        dst[c] = ap;
        acc[0] = fma(own[c], ap, acc[0]);
      }
      if (MODE == H3_DIR) {
        double *pn = pnew + 3 * n;
#pragma unroll
        for (int c = 0; c < 3; ++c) pn[c] = own[c];
      }
    } else if (MODE == H3_RES) {
      // fixed rows of K are identity rows: (K u)_fixed = u_fixed
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double ku = ((fm >> c) & 1u) ? own[c] : o[c];
        const double r = a.f[3 * n + c] - ku;
        dst[c] = r;
        double z = r;
        if (PRE == TPO_PRECOND_JACOBI) {
          z = r / a.diag[3 * n + c];
          a.z[3 * n + c] = z;
        }
        acc[0] = fma(r, z, acc[0]);
        acc[1] = fma(r, r, acc[1]);
      }
    } else {  // H3_BLOCK
      const double s = inv_sqrt_count(g, p.ix, p.iy, p.iz);
      const double *r = a.x + 3 * n;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double z = ((fm >> c) & 1u) ? 0.0 : o[c] * s;
        dst[c] = z;
        acc[0] = fma(r[c], z, acc[0]);
        acc[1] = fma(r[c], r[c], acc[1]);
      }
    }
  }
  uint32_t *counter = MODE == H3_APPLY ? a.counter : &ctl->counter;
  if (!grid_reduce<2>(acc, a.part, counter)) return;
  if (threadIdx.x != 0) return;
  if (MODE == H3_APPLY) {
    if (a.pap_out) *a.pap_out = acc[0];
  } else if (MODE == H3_DIR) {
    const double pap = acc[0];
    ctl->pap = pap;
    ctl->first = 0;
    if (!finite(pap)) ctl->status = TPO_SOLVE_NONFINITE;
    else if (fabs(pap) < 1e-30) ctl->status = TPO_SOLVE_BREAKDOWN;  // solver.py:114-115
    else ctl->alpha = ctl->rz / pap;                                  // solver.py:117
  } else if (MODE == H3_RES || a.init) {
    ctl->it = 0;
    ctl->first = 1;
    ctl->rz = acc[0];
    ctl->rr = acc[1];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  } else {
    finish_update(ctl, acc[0], acc[1]);
  }
}

// ---------------------------------------------------------------------------
// Plane-marching form of the same gathers. A CTA owns HT_THREADS consecutive
// nodes j0 .. j0+T-1 of a y-z plane (plane index j = iy*(nelz+1) + iz, one
// node per thread) and walks them along x over a chunk of planes. Node
// values (direction: p' = z + beta p, formed ONCE per node) are staged per
// plane in shared memory for the run j0-(nelz+2) .. j0+T+nelz+1, which holds
// every y/z neighbour of the CTA's nodes, in a ring of three planes (x-1, x,
// x+1); element weights in a ring of three element planes. The 27-point
// gather reads shared memory.
// Neighbours that wrap around a z-row are never used with a nonzero weight:
// every element containing them lies outside the grid, and those weights are
// zero.
// Pipelining: while plane x is computed, plane x+2's node values (raw, as
// they lie in memory: a contiguous run per plane) and element plane x+1 are
// already on their way into shared memory by cp.async; at the next step the
// raw run is turned into the ring's layout (p' = z + beta p, or the
// element-block scaling). Two barriers per plane; no global load waits in the
// compute loop. Layout of the dynamic shared memory (doubles):
//   nodes  [3 planes][3 components][NH],  NH = T + 2*(nelz+2)
//   raw    [2 arrays][3*NH]               (z and p for the direction)
//   elems  [3 planes][EH],                EH = T + nelz + 2
// ---------------------------------------------------------------------------
constexpr int HT_THREADS = 256;

__host__ __device__ inline int hex_tile_nh(int nz) { return HT_THREADS + 2 * (nz + 2); }
__host__ __device__ inline int hex_tile_eh(int nz) { return HT_THREADS + nz + 2; }
__host__ __device__ inline size_t hex_tile_smem(int nz) {
  return (size_t)(15 * hex_tile_nh(nz) + 3 * hex_tile_eh(nz)) * sizeof(double);
}

// 8-byte asynchronous global -> shared copy (no register staging)
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// At most 80 registers: three CTAs (24 warps) per SM hide the barriers and
// the shared-memory latency better than two CTAs at 110 registers, for a few
// bytes of spill (52.1 vs 56.1 us per direction launch at 128x64x64).
template <int MODE, int PRE>
__global__ void __launch_bounds__(HT_THREADS, 3) k_hex_tile(Hex3Args a, int xc) {
  PcgCtl *ctl = a.ctl;
  if (MODE != H3_APPLY && ctl->status != TPO_SOLVE_RUNNING) return;
  extern __shared__ double hs[];
  const Hex3 g = a.g;
  const int nz1 = g.nz + 1;
  const int64_t P = (int64_t)(g.ny + 1) * nz1;  // nodes per x-plane
  const int64_t PE = (int64_t)g.ny * g.nz;      // elements per x-plane
  const int NH = hex_tile_nh(g.nz), EH = hex_tile_eh(g.nz);
  double *sv = hs;            // node ring
  double *sr = hs + 9 * NH;   // raw node run(s) of the next plane
  double *se = sr + 6 * NH;   // element ring
  const int64_t j0 = (int64_t)blockIdx.x * HT_THREADS;
  const int xa = blockIdx.y * xc, xb = min(xa + xc, g.nx + 1);
  const int64_t j = j0 + threadIdx.x;
  const bool mine = j < P;
  const int iy = (int)(j / nz1), iz = (int)(j - (int64_t)iy * nz1);
  const int iy0 = (int)(j0 / nz1), iz0 = (int)(j0 - (int64_t)iy0 * nz1);
  const int64_t kmin = (int64_t)(iy0 - 1) * g.nz + (iz0 - 1);  // first staged element
  const int hoff = g.nz + 2;                                  // halo before j0

  bool first = true;
  double beta = 0.0;
  const double *pold = nullptr;
  double *pnew = nullptr;
  if (MODE == H3_DIR) {
    first = ctl->first != 0;
    beta = ctl->beta;
    const bool odd = ctl->it & 1;
    pold = odd ? a.pb : a.pa;
    pnew = odd ? a.pa : a.pb;
  }

  const int64_t jA = j0 - hoff;  // first staged plane index
  const bool two = MODE == H3_DIR && !first;
  // node plane x: its raw run (z and p for the direction) -> sr, by cp.async
  auto issue_nodes = [&](int x) {
    const bool xin = x >= 0 && x <= g.nx;
    for (int t = threadIdx.x; t < 3 * NH; t += HT_THREADS) {
      const int64_t jj = jA + t / 3;
      if (xin && jj >= 0 && jj < P) {
        const int64_t off = 3 * ((int64_t)x * P + jA) + t;
        cp_async8(sr + t, a.x + off);
        if (two) cp_async8(sr + 3 * NH + t, pold + off);
      } else {
        sr[t] = 0.0;
        if (two) sr[3 * NH + t] = 0.0;
      }
    }
  };
  // element plane ex -> element slot (ex + 3) % 3, by cp.async
  auto issue_elems = [&](int ex) {
    double *d = se + ((ex + 3) % 3) * EH;
    const bool xin = ex >= 0 && ex < g.nx;
    for (int i = threadIdx.x; i < EH; i += HT_THREADS) {
      const int64_t k = kmin + i;
      if (xin && k >= 0 && k < PE) cp_async8(d + i, a.w + (int64_t)ex * PE + k);
      else d[i] = 0.0;
    }
  };
  // raw run of node plane x -> node slot (x + 3) % 3 (component-major)
  auto combine = [&](int x) {
    double *d = sv + ((x + 3) % 3) * 3 * NH;
    for (int i = threadIdx.x; i < NH; i += HT_THREADS) {
      double v[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = sr[3 * i + c];
      const int64_t jj = jA + i;
      if (MODE == H3_DIR) {
        if (two) {
#pragma unroll
          for (int c = 0; c < 3; ++c) v[c] = fma(beta, sr[3 * NH + 3 * i + c], v[c]);
        }
        // the CTA's own nodes: store the new direction once
        if (x >= xa && x < xb && i >= hoff && i < hoff + HT_THREADS && jj < P) {
          double *pn = pnew + 3 * ((int64_t)x * P + jj);
#pragma unroll
          for (int c = 0; c < 3; ++c) pn[c] = v[c];
        }
      }
      if (MODE == H3_BLOCK && x >= 0 && x <= g.nx && jj >= 0 && jj < P) {
        const int my = (int)(jj / nz1), mz = (int)(jj - (int64_t)my * nz1);
        const double sc = inv_sqrt_count(g, x, my, mz);
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] *= sc;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) d[c * NH + i] = v[c];
    }
  };

  // prologue: planes xa-1 and xa staged, plane xa+1 and element plane xa in flight
  issue_nodes(xa - 1);
  issue_elems(xa - 1);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  combine(xa - 1);
  __syncthreads();
  issue_nodes(xa);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  combine(xa);
  __syncthreads();
  issue_nodes(xa + 1);
  issue_elems(xa);
  cp_async_commit();
  double acc[2] = {0.0, 0.0};
  const int c0 = (int)(j - j0) + hoff;  // this node's slot in a staged plane
  for (int x = xa; x < xb; ++x) {
    cp_async_wait_all();
    __syncthreads();  // raw = node plane x+1, element slot x%3 = element plane x
    combine(x + 1);
    __syncthreads();  // node slot (x+1)%3 complete, raw free
    if (x + 1 < xb) {
      issue_nodes(x + 2);
      issue_elems(x + 1);
      cp_async_commit();
    }
    if (mine) {
      const double *pl[3] = {sv + ((x + 2) % 3) * 3 * NH, sv + (x % 3) * 3 * NH,
                             sv + ((x + 1) % 3) * 3 * NH};
      const double *el[2] = {se + ((x + 2) % 3) * EH, se + (x % 3) * EH};
      double we[8];
#pragma unroll
      for (int ex = 0; ex < 2; ++ex)
#pragma unroll
        for (int ey = 0; ey < 2; ++ey)
#pragma unroll
          for (int ez = 0; ez < 2; ++ez) {
            const int y = iy - 1 + ey, z = iz - 1 + ez;
            const bool ok = y >= 0 && y < g.ny && z >= 0 && z < g.nz;
            we[(ex * 2 + ey) * 2 + ez] = ok ? el[ex][(int64_t)y * g.nz + z - kmin] : 0.0;
          }
      double own[3] = {0.0, 0.0, 0.0};
      auto load = [&](int ox, int oy, int oz, double (&v)[3]) {
        const double *src = pl[ox + 1] + c0 + oy * nz1 + oz;
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = src[c * NH];
        if (ox == 0 && oy == 0 && oz == 0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) own[c] = v[c];
        }
      };
      double o[3];
      hex_gather<MODE == H3_BLOCK>(we, load, o);
      const int64_t n = (int64_t)x * P + j;
      const unsigned fm = a.mask[n];
      double *dst = a.out + 3 * n;
      if (MODE == H3_APPLY || MODE == H3_DIR) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double ap = ((fm >> c) & 1u) ? own[c] : o[c];
          dst[c] = ap;
          acc[0] = fma(own[c], ap, acc[0]);
        }
      } else if (MODE == H3_RES) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double ku = ((fm >> c) & 1u) ? own[c] : o[c];
          const double r = a.f[3 * n + c] - ku;
          dst[c] = r;
          double z = r;
          if (PRE == TPO_PRECOND_JACOBI) {
            z = r / a.diag[3 * n + c];
            a.z[3 * n + c] = z;
          }
          acc[0] = fma(r, z, acc[0]);
          acc[1] = fma(r, r, acc[1]);
        }
      } else {  // H3_BLOCK
        const double s = inv_sqrt_count(g, x, iy, iz);
        const double *r = a.x + 3 * n;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double z = ((fm >> c) & 1u) ? 0.0 : o[c] * s;
          dst[c] = z;
          acc[0] = fma(r[c], z, acc[0]);
          acc[1] = fma(r[c], r[c], acc[1]);
        }
      }
    }
  }
  cp_async_wait_all();
  uint32_t *counter = MODE == H3_APPLY ? a.counter : &ctl->counter;
  if (!grid_reduce<2>(acc, a.part, counter)) return;
  if (threadIdx.x != 0) return;
  if (MODE == H3_APPLY) {
    if (a.pap_out) *a.pap_out = acc[0];
  } else if (MODE == H3_DIR) {
    const double pap = acc[0];
    ctl->pap = pap;
    ctl->first = 0;
    if (!finite(pap)) ctl->status = TPO_SOLVE_NONFINITE;
    else if (fabs(pap) < 1e-30) ctl->status = TPO_SOLVE_BREAKDOWN;  // solver.py:114-115
    else ctl->alpha = ctl->rz / pap;                                  // solver.py:117
  } else if (MODE == H3_RES || a.init) {
    ctl->it = 0;
    ctl->first = 1;
    ctl->rz = acc[0];
    ctl->rr = acc[1];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  } else {
    finish_update(ctl, acc[0], acc[1]);
  }
}

// ---------------------------------------------------------------------------
// Structured H8 operator. For the unit-cube trilinear element of an isotropic
// material with exact (2x2x2 Gauss) integration, f = w Ke u follows from the
// element's trilinear modal coefficients:
// * an 8-point Walsh-Hadamard transform maps each displacement component's
//   corner values onto the monomials 1, xi, eta, zeta, xi eta, eta zeta,
//   zeta xi, xi eta zeta;
// * the monomials are orthogonal under the element integral, so the strain
//   energy splits into the constant gradient (an isotropic stress), three
//   linear-gradient groups and one bilinear group, a few multiply-adds each;
// * the modal forces return to the corners by the transposed transform.
// About 180 FP64 operations instead of the 576 multiply-adds of the dense
// 24x24 product. Corner arrays are indexed by bits dx + 2 dy + 4 dz; modal
// index m = mx + 2 my + 4 mz is the monomial xi^mx eta^my zeta^mz.
// The constants include the 1/64 of the two unnormalised transforms:
//   L4 = 4 lam, M8 = 8 mu, M4 = 4 mu, A = 4 lam / 3, Cc = 4 mu / 3,
//   K2 = 4 (lam + 4 mu) / 9, all / 64.
struct H8Const {
  double L4, M8, M4, A, Cc, K2;
};
__constant__ H8Const c_h8s;

__host__ __device__ inline H8Const h8_const(double lam, double mu) {
  const double q = 1.0 / 64.0;
  return H8Const{4.0 * lam * q, 8.0 * mu * q, 4.0 * mu * q, (4.0 / 3.0) * lam * q,
                 (4.0 / 3.0) * mu * q, (4.0 / 9.0) * (lam + 4.0 * mu) * q};
}

__host__ __device__ inline void h8_forces(const H8Const &k, double w, const double (&v)[8][3],
                                          double (&f)[8][3]) {
  double c[8][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = v[i][j];
#pragma unroll
    for (int b = 1; b < 8; b <<= 1)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (!(i & b)) {
          const double lo = t[i], hi = t[i + b];
          t[i] = lo + hi;  // modal bit 0: the sum
          t[i + b] = hi - lo;  // modal bit 1: + at the corner whose bit is 1
        }
#pragma unroll
    for (int i = 0; i < 8; ++i) c[i][j] = t[i];
  }
  const double L4 = w * k.L4, M8 = w * k.M8, M4 = w * k.M4;
  const double A = w * k.A, Cc = w * k.Cc, K2 = w * k.K2;
  // constant gradient: columns xi (m=1), eta (m=2), zeta (m=4)
  const double *a = c[1], *b = c[2], *d = c[4];
  const double ltr = L4 * (a[0] + b[1] + d[2]);
  const double nx = fma(M8, a[0], ltr), ny = fma(M8, b[1], ltr), nz = fma(M8, d[2], ltr);
  const double sxy = M4 * (a[1] + b[0]), sxz = M4 * (a[2] + d[0]), syz = M4 * (b[2] + d[1]);
  // linear gradients: xi eta (m=3), eta zeta (m=6), zeta xi (m=5)
  const double *p = c[3], *q = c[6], *r = c[5];
  const double Te = A * (p[0] + q[2]), Tx = A * (p[1] + r[2]), Tz = A * (r[0] + q[1]);
  const double W = (p[2] + r[1]) + q[0];
  double F[8][3];
  F[0][0] = F[0][1] = F[0][2] = 0.0;
  F[1][0] = nx;  F[1][1] = sxy; F[1][2] = sxz;
  F[2][0] = sxy; F[2][1] = ny;  F[2][2] = syz;
  F[4][0] = sxz; F[4][1] = syz; F[4][2] = nz;
  F[3][0] = fma(M4, p[0], Te); F[3][1] = fma(M4, p[1], Tx); F[3][2] = Cc * (W + p[2]);
  F[6][0] = Cc * (W + q[0]);   F[6][1] = fma(M4, q[1], Tz); F[6][2] = fma(M4, q[2], Te);
  F[5][0] = fma(M4, r[0], Tz); F[5][1] = Cc * (W + r[1]);   F[5][2] = fma(M4, r[2], Tx);
  // bilinear: xi eta zeta (m=7)
  F[7][0] = K2 * c[7][0]; F[7][1] = K2 * c[7][1]; F[7][2] = K2 * c[7][2];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = F[i][j];
#pragma unroll
    for (int b2 = 1; b2 < 8; b2 <<= 1)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (!(i & b2)) {
          const double lo = t[i], hi = t[i + b2];
          t[i] = lo - hi;      // corner bit 0: - the odd monomial
          t[i + b2] = lo + hi;  // corner bit 1: +
        }
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i][j] = t[i];
  }
}

// ---------------------------------------------------------------------------
// Element-centric plane march with the structured operator (matvec, direction
// and residual modes; the element-block preconditioner keeps the dense
// gather). A CTA owns a y-z tile of EY x EZ elements, one per thread, whose
// origins are (y0 - 1 + ey, z0 - 1 + ez), and the (EY-1) x (EZ-1) nodes
// (y0 + ey, z0 + ez) in it; it walks node planes xa .. xb-1 along x.
// * Node planes are staged HE_DEPTH ahead by cp.async into a ring of raw
//   slots: a slot holds one node plane's run (the values, and for the
//   direction the previous direction too) and the weights of the element
//   plane before it, one cp.async group per plane.
// * Each thread reads its element's four corners in node plane x+1 from the
//   ring, forming the direction p' = z + beta p there (a node's value is
//   formed by each of its four elements, in the same arithmetic; the thread
//   whose node it is stores it). Its corners in plane x are kept from the
//   step before.
// * A thread computes its element of element plane x (between node planes x
//   and x+1) and keeps the two corners at its own node. The six other
//   corners that nodes of the tile need are handed over in shared memory.
// * A node then adds, in a fixed order, the dx = 0 corners of its four
//   elements in element plane x and the dx = 1 corners carried from element
//   plane x-1, and is finished. Each chunk of planes starts with element
//   plane xa-1 (its dx = 1 corners only).
// Two barriers per plane; no atomics; the summation order is fixed.
// Shared memory (doubles): raw ring [HE_DEPTH][6 NS + HE_THREADS]; handover
// [18][HE_THREADS]; NS = (EY + 1)(EZ + 1).
// ---------------------------------------------------------------------------
constexpr int HE_THREADS = 256;
constexpr int HE_DEPTH = 3;
constexpr int HE_KS = 6;  // staged values per thread and plane: 3 NS <= HE_KS * HE_THREADS
__host__ __device__ inline int hex_elem_ns(int EY, int EZ) { return (EY + 1) * (EZ + 1); }
__host__ __device__ inline int hex_elem_rs(int EY, int EZ) {
  return 6 * hex_elem_ns(EY, EZ) + HE_THREADS;
}
__host__ __device__ inline size_t hex_elem_smem(int EY, int EZ) {
  return (size_t)(HE_DEPTH * hex_elem_rs(EY, EZ) + 18 * HE_THREADS) * sizeof(double);
}
template <int N> __device__ __forceinline__ void cp_async_wait_pending() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int MODE, int PRE>
__global__ void __launch_bounds__(HE_THREADS, 2)
    k_hex_elem(Hex3Args a, int EY, int EZ, int tzc, int xc) {
  static_assert(MODE != H3_BLOCK, "the element-block preconditioner uses the dense gather");
  static_assert(HE_DEPTH >= 2, "the prologue waits for two staged planes");
  PcgCtl *ctl = a.ctl;
  if (MODE != H3_APPLY && ctl->status != TPO_SOLVE_RUNNING) return;
  extern __shared__ double hs[];
  const Hex3 g = a.g;
  const int NS = hex_elem_ns(EY, EZ), RS = hex_elem_rs(EY, EZ);
  const int RW = EZ + 1;                   // staged nodes per y-row
  double *sring = hs;                      // raw ring
  double *sx = sring + HE_DEPTH * RS;      // handover
  const int ty = (int)blockIdx.x / tzc, tz = (int)blockIdx.x - ty * tzc;
  const int y0 = ty * (EY - 1), z0 = tz * (EZ - 1);
  const int xa = blockIdx.y * xc, xb = min(xa + xc, g.nx + 1);
  const int t = threadIdx.x;
  const bool el = t < EY * EZ;
  const int ey = el ? t / EZ : 0, ez = el ? t - (t / EZ) * EZ : 0;
  const int Y = y0 - 1 + ey, Z = z0 - 1 + ez;  // element origin
  const bool eyz = el && Y >= 0 && Y < g.ny && Z >= 0 && Z < g.nz;
  const int oy = y0 + ey, oz = z0 + ez;        // the node this thread finishes
  const bool owner = el && ey < EY - 1 && ez < EZ - 1 && oy <= g.ny && oz <= g.nz;
  const int64_t ny1 = g.ny + 1, nz1 = g.nz + 1;
  const int64_t P1 = ny1 * nz1, P3 = 3 * P1;  // nodes, values per node plane
  const int64_t own0 = (int64_t)oy * nz1 + oz;  // plane-relative index of the own node

  bool first = true;
  double beta = 0.0;
  const double *pold = nullptr;
  double *pnew = nullptr;
  if (MODE == H3_DIR) {
    first = ctl->first != 0;
    beta = ctl->beta;
    const bool odd = ctl->it & 1;
    pold = odd ? a.pb : a.pa;
    pnew = odd ? a.pa : a.pb;
  }
  const bool two = MODE == H3_DIR && !first;

  // The staging pattern is the same in every plane: each thread's values as
  // plane-relative offsets into the node arrays (-1 outside the grid). A
  // plane has at most 2^29 nodes (grid <= 2^30 nodes, >= 2 planes), so the
  // offsets fit 32 bits.
  int goff[HE_KS];
#pragma unroll
  for (int k = 0; k < HE_KS; ++k) {
    const int i = t + k * HE_THREADS;
    const int li = i / 3;
    const int iyl = li / RW, izl = li - iyl * RW;
    const int y = y0 - 1 + iyl, z = z0 - 1 + izl;
    goff[k] = (i < 3 * NS && y >= 0 && y <= g.ny && z >= 0 && z <= g.nz)
                  ? 3 * (y * (int)nz1 + z) + (i - 3 * li)
                  : -1;
  }

  auto slot_of = [&](int x) { return sring + ((x + 3 * HE_DEPTH) % HE_DEPTH) * RS; };
  // raw run of node plane x and the weights of element plane x-1 -> its ring
  // slot (3 values per node, as in memory), one cp.async group
  auto issue = [&](int x) {
    if (x <= xb) {  // planes past xb are not needed
      double *sr = slot_of(x);
      const bool xin = x >= 0 && x <= g.nx;
      if (el) {
        const int ex = x - 1;
        if (eyz && ex >= 0 && ex < g.nx)
          cp_async8(sr + 6 * NS + t, a.w + ((int64_t)ex * g.ny + Y) * g.nz + Z);
        else
          sr[6 * NS + t] = 0.0;
      }
      const double *bx = a.x + (int64_t)x * P3;
      const double *bp = two ? pold + (int64_t)x * P3 : nullptr;
#pragma unroll
      for (int k = 0; k < HE_KS; ++k) {
        const int i = t + k * HE_THREADS;
        if (i >= 3 * NS) break;
        if (xin && goff[k] >= 0) {
          cp_async8(sr + i, bx + goff[k]);
          if (two) cp_async8(sr + 3 * NS + i, bp + goff[k]);
        } else {
          sr[i] = 0.0;
          if (two) sr[3 * NS + i] = 0.0;
        }
      }
    }
    cp_async_commit();
  };
  // this thread's element corners (dy, dz) in node plane x, [dy + 2 dz][c],
  // formed from the raw run; the direction's own node is stored once
  auto corners = [&](int x, double (&q)[4][3]) {
    const double *sr = slot_of(x) + 3 * (ey * RW + ez);
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int o = 3 * (dy * RW + dz) + c;
          q[dy + 2 * dz][c] = two ? fma(beta, sr[3 * NS + o], sr[o]) : sr[o];
        }
    if (MODE == H3_DIR && owner && x >= xa && x < xb) {
      double *pn = pnew + (int64_t)x * P3 + 3 * own0;
#pragma unroll
      for (int c = 0; c < 3; ++c) pn[c] = q[3][c];
    }
  };
  auto weight_of = [&](int x) { return el ? slot_of(x)[6 * NS + t] : 0.0; };  // element plane x-1
  // element forces from corners in planes x (lo) and x+1 (hi); the six
  // corners other nodes take go to the handover arrays, the two at this
  // thread's node stay: own[dx][c]
  auto element = [&](const double (&lo)[4][3], const double (&hi)[4][3], double w,
                     double (&own)[2][3]) {
    double v[8][3], f[8][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        v[2 * k][c] = lo[k][c];      // bit dx = 0; k = dy + 2 dz -> bits 2 dy + 4 dz
        v[2 * k + 1][c] = hi[k][c];  // dx = 1
      }
    h8_forces(c_h8s, w, v, f);
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sx[((0 * 2 + dx) * 3 + c) * HE_THREADS + t] = f[dx + 4][c];  // corner (0,1): node (ey-1, ez)
        sx[((1 * 2 + dx) * 3 + c) * HE_THREADS + t] = f[dx + 2][c];  // corner (1,0): node (ey, ez-1)
        sx[((2 * 2 + dx) * 3 + c) * HE_THREADS + t] = f[dx + 0][c];  // corner (0,0): node (ey-1, ez-1)
        own[dx][c] = f[dx + 6][c];                                   // corner (1,1): this node
      }
  };
  // this node's sum over its four elements of element plane x, corner dx
  const int tA = (ey + 1) * EZ + ez, tB = ey * EZ + ez + 1, tC = (ey + 1) * EZ + ez + 1;
  auto gather = [&](const double (&own)[2][3], int dx, double (&s)[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      s[c] = ((own[dx][c] + sx[((0 * 2 + dx) * 3 + c) * HE_THREADS + tA]) +
              sx[((1 * 2 + dx) * 3 + c) * HE_THREADS + tB]) +
             sx[((2 * 2 + dx) * 3 + c) * HE_THREADS + tC];
  };

  // prologue: node planes xa-1 .. xa-2+HE_DEPTH in flight; element plane
  // xa-1 from planes xa-1 and xa, its dx = 1 corners carried into node plane
  // xa. A ring slot is refilled (plane x + HE_DEPTH into the slot of plane
  // x) once every thread has read plane x.
  for (int k = 0; k < HE_DEPTH; ++k) issue(xa - 1 + k);
  cp_async_wait_pending<HE_DEPTH - 2>();
  __syncthreads();  // planes xa-1 and xa landed
  double cur[4][3] = {}, nxt[4][3] = {}, own[2][3] = {}, carry[3] = {0.0, 0.0, 0.0};
  unsigned fm = owner ? a.mask[(int64_t)xa * P1 + own0] : 0u;
  if (el) {
    corners(xa - 1, cur);
    corners(xa, nxt);
    element(cur, nxt, weight_of(xa), own);
  }
  __syncthreads();  // handover of element plane xa-1 complete; planes xa-1, xa read
  if (owner) gather(own, 1, carry);
  issue(xa - 1 + HE_DEPTH);
  issue(xa + HE_DEPTH);
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) cur[k][c] = nxt[k][c];

  double acc[2] = {0.0, 0.0};
  for (int x = xa; x < xb; ++x) {
    cp_async_wait_pending<HE_DEPTH - 1>();
    __syncthreads();  // plane x+1 landed; every thread is done with the handover
    // the mask of this thread's node in plane x+1, for the next step
    const unsigned fm_next = (owner && x + 1 < xb) ? a.mask[(int64_t)(x + 1) * P1 + own0] : 0u;
    if (el) {
      corners(x + 1, nxt);
      element(cur, nxt, weight_of(x + 1), own);
    }
    __syncthreads();  // handover of element plane x complete; plane x+1 read
    issue(x + 1 + HE_DEPTH);
    if (owner) {
      double s0[3], s1[3];
      gather(own, 0, s0);
      gather(own, 1, s1);
      double o[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        o[c] = carry[c] + s0[c];
        carry[c] = s1[c];
      }
      // this node's own value in plane x: its element's corner (dx, dy, dz) = (0, 1, 1)
      const double *self = cur[3];
      const int64_t n = (int64_t)x * P1 + own0;
      double *dst = a.out + 3 * n;
      if (MODE == H3_APPLY || MODE == H3_DIR) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double ap = ((fm >> c) & 1u) ? self[c] : o[c];
          dst[c] = ap;
          acc[0] = fma(self[c], ap, acc[0]);
        }
      } else {  // H3_RES
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double ku = ((fm >> c) & 1u) ? self[c] : o[c];
          const double r = a.f[3 * n + c] - ku;
          dst[c] = r;
          double zz = r;
          if (PRE == TPO_PRECOND_JACOBI) {
            zz = r / a.diag[3 * n + c];
            a.z[3 * n + c] = zz;
          }
          acc[0] = fma(r, zz, acc[0]);
          acc[1] = fma(r, r, acc[1]);
        }
      }
    }
    fm = fm_next;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) cur[k][c] = nxt[k][c];
  }
  cp_async_wait_all();
  uint32_t *counter = MODE == H3_APPLY ? a.counter : &ctl->counter;
  if (!grid_reduce<2>(acc, a.part, counter)) return;
  if (threadIdx.x != 0) return;
  if (MODE == H3_APPLY) {
    if (a.pap_out) *a.pap_out = acc[0];
  } else if (MODE == H3_DIR) {
    const double pap = acc[0];
    ctl->pap = pap;
    ctl->first = 0;
    if (!finite(pap)) ctl->status = TPO_SOLVE_NONFINITE;
    else if (fabs(pap) < 1e-30) ctl->status = TPO_SOLVE_BREAKDOWN;  // solver.py:114-115
    else ctl->alpha = ctl->rz / pap;                                  // solver.py:117
  } else {
    ctl->it = 0;
    ctl->first = 1;
    ctl->rz = acc[0];
    ctl->rr = acc[1];
    if (!finite(acc[0]) || !finite(acc[1])) ctl->status = TPO_SOLVE_NONFINITE;
  }
}

// ---------------------------------------------------------------------------
// Pointwise kernels
// ---------------------------------------------------------------------------
// u += alpha p', r -= alpha ap; Jacobi / none: z = r / diag (or r), r.z,
// ||r||^2 and the stop / beta decision. Element-block: u and r only (the
// preconditioner kernel that follows reduces and decides).
template <int PRE>
__global__ void __launch_bounds__(H3_FLAT)
    k_hex_update(int64_t ndof, double *__restrict__ u, double *__restrict__ r,
                 const double *__restrict__ pa, const double *__restrict__ pb,
                 const double *__restrict__ ap, const double *__restrict__ diag,
                 double *__restrict__ z, double *part, PcgCtl *ctl) {
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const double alpha = ctl->alpha;
  const double *__restrict__ p = (ctl->it & 1) ? pa : pb;  // written by this iteration's direction
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndof;
       i += (int64_t)gridDim.x * blockDim.x) {
    u[i] = fma(alpha, p[i], u[i]);
    const double rn = fma(-alpha, ap[i], r[i]);
    r[i] = rn;
    if (PRE != TPO_PRECOND_BLOCK_JACOBI) {
      double zn = rn;
      if (PRE == TPO_PRECOND_JACOBI) {
        zn = rn / diag[i];
        z[i] = zn;
      }
      acc[0] = fma(rn, zn, acc[0]);
      acc[1] = fma(rn, rn, acc[1]);
    }
  }
  if (PRE == TPO_PRECOND_BLOCK_JACOBI) return;
  if (!grid_reduce<2>(acc, part, &ctl->counter)) return;
  if (threadIdx.x == 0) finish_update(ctl, acc[0], acc[1]);
}

// The same update with 16-byte loads and stores, two DOFs per thread and
// step (every array 16-byte aligned; the host checks). An odd last DOF is
// taken by the thread that would hold its pair.
template <int PRE>
__global__ void __launch_bounds__(H3_FLAT)
    k_hex_update2(int64_t ndof, double *__restrict__ u, double *__restrict__ r,
                  const double *__restrict__ pa, const double *__restrict__ pb,
                  const double *__restrict__ ap, const double *__restrict__ diag,
                  double *__restrict__ z, double *part, PcgCtl *ctl) {
  if (ctl->status != TPO_SOLVE_RUNNING) return;
  const double alpha = ctl->alpha;
  const double *__restrict__ p = (ctl->it & 1) ? pa : pb;  // written by this iteration's direction
  double acc[2] = {0.0, 0.0};
  auto one = [&](double uu, double pp, double aa, double rr, double dd, double &uo, double &ro,
                 double &zo) {
    uo = fma(alpha, pp, uu);
    ro = fma(-alpha, aa, rr);
    if (PRE != TPO_PRECOND_BLOCK_JACOBI) {
      zo = PRE == TPO_PRECOND_JACOBI ? ro / dd : ro;
      acc[0] = fma(ro, zo, acc[0]);
      acc[1] = fma(ro, ro, acc[1]);
    }
  };
  const int64_t npair = ndof / 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= npair;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (k < npair) {
      const double2 uu = reinterpret_cast<const double2 *>(u)[k];
      const double2 pp = reinterpret_cast<const double2 *>(p)[k];
      const double2 aa = reinterpret_cast<const double2 *>(ap)[k];
      const double2 rr = reinterpret_cast<const double2 *>(r)[k];
      const double2 dd = PRE == TPO_PRECOND_JACOBI ? reinterpret_cast<const double2 *>(diag)[k]
                                                   : make_double2(1.0, 1.0);
      double2 uo, ro, zo;
      one(uu.x, pp.x, aa.x, rr.x, dd.x, uo.x, ro.x, zo.x);
      one(uu.y, pp.y, aa.y, rr.y, dd.y, uo.y, ro.y, zo.y);
      reinterpret_cast<double2 *>(u)[k] = uo;
      reinterpret_cast<double2 *>(r)[k] = ro;
      if (PRE == TPO_PRECOND_JACOBI) reinterpret_cast<double2 *>(z)[k] = zo;
    } else if (ndof & 1) {  // k == npair: the odd last DOF
      const int64_t i = ndof - 1;
      double uo, ro, zo;
      one(u[i], p[i], ap[i], r[i], PRE == TPO_PRECOND_JACOBI ? diag[i] : 1.0, uo, ro, zo);
      u[i] = uo;
      r[i] = ro;
      if (PRE == TPO_PRECOND_JACOBI) z[i] = zo;
    }
  }
  if (PRE == TPO_PRECOND_BLOCK_JACOBI) return;
  if (!grid_reduce<2>(acc, part, &ctl->counter)) return;
  if (threadIdx.x == 0) finish_update(ctl, acc[0], acc[1]);
}

// SIMP scales s = e_min + rho^p (1 - e_min) (reference fem/kernels.py:92) and,
// for the element-block preconditioner, w = s / max(s, alpha)^2
// (preconditioner.py:128-130).
__global__ void k_hex_scales(int64_t ne, const double *__restrict__ rho, double e_min, double pen,
                             double alpha_reg, double *__restrict__ s, double *__restrict__ w) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double v = e_min + pow(rho[e], pen) * (1.0 - e_min);
    s[e] = v;
    if (w) {
      const double sc = fmax(v, alpha_reg);
      w[e] = v / (sc * sc);
    }
  }
}

// Jacobi diagonal: sum_e s_e Ke_ii over the node's elements; fixed -> 1,
// floor 1e-20 (reference fem/kernels.py:104-129).
__global__ void k_hex_diag(Hex3 g, const double *__restrict__ s, const uint8_t *__restrict__ mask,
                           double *__restrict__ diag) {
  const int64_t total = g.nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < total;
       n += (int64_t)gridDim.x * blockDim.x) {
    const NodePos p = node_pos(g, n);
    double we[8];
    node_elem_weights(g, p, s, we);
    const unsigned fm = mask[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double d = 0.0;
#pragma unroll
      for (int ex = 0; ex < 2; ++ex)
#pragma unroll
        for (int ey = 0; ey < 2; ++ey)
#pragma unroll
          for (int ez = 0; ez < 2; ++ez) {
            const int a = h8_corner(1 - ex, 1 - ey, 1 - ez);
            d = fma(we[(ex * 2 + ey) * 2 + ez], c_ke3[(3 * a + c) * 25], d);
          }
      if ((fm >> c) & 1u) d = 1.0;
      else if (d < 1e-20) d = 1e-20;
      diag[3 * n + c] = d;
    }
  }
}

// Warm start: fixed DOFs of u are zeroed (reference solver.py:52-57).
__global__ void k_hex_zero_fixed(int64_t nn, const uint8_t *__restrict__ mask, double *u) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const unsigned fm = mask[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((fm >> c) & 1u) u[3 * n + c] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Compliance and sensitivity, one element per thread (reference
// fem/kernels.py:275-308): uKu_e = u_e^T Ke u_e, dc_e = -p rho^(p-1)(1-e_min) uKu_e,
// c = sum_e (e_min + rho^p (1 - e_min)) uKu_e.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(H3_THREADS)
    k_hex_sensitivity(Hex3 g, double e_min, double pen, const double *__restrict__ rho,
                      const double *__restrict__ u, double *__restrict__ dc, double *part,
                      SumCtl *ctl, double *c_out) {
  const int64_t ne = g.elems();
  const int64_t sy = g.nz + 1, sx = (int64_t)(g.ny + 1) * sy;
  double acc[1] = {0.0};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = e / g.nz;
    const int ez = (int)(e - col * g.nz);
    const int ex = (int)(col / g.ny);
    const int ey = (int)(col - (int64_t)ex * g.ny);
    const int64_t n0 = (int64_t)ex * sx + (int64_t)ey * sy + ez;
    double ue[24];
#pragma unroll
    for (int dx = 0; dx < 2; ++dx)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dz = 0; dz < 2; ++dz) {
          const int b = h8_corner(dx, dy, dz);
          const double *src = u + 3 * (n0 + dx * sx + dy * sy + dz);
#pragma unroll
          for (int j = 0; j < 3; ++j) ue[3 * b + j] = src[j];
        }
    double uku = 0.0;
#pragma unroll
    for (int i = 0; i < 24; ++i) {
      double ku = c_ke3[i * 24] * ue[0];
#pragma unroll
      for (int j = 1; j < 24; ++j) ku = fma(c_ke3[i * 24 + j], ue[j], ku);
      uku = fma(ue[i], ku, uku);
    }
    const double r = rho[e];
    dc[e] = -pen * pow(r, pen - 1.0) * (1.0 - e_min) * uku;
    acc[0] += (e_min + pow(r, pen) * (1.0 - e_min)) * uku;
  }
  if (!grid_reduce<1>(acc, part, &ctl->counter)) return;
  if (threadIdx.x == 0) *c_out = acc[0];
}

// ---------------------------------------------------------------------------
// Hat-weight filters over the 3D box |dx|,|dy|,|dz| <= R = ceil(rmin)
// (reference optimizer/filter.py:75-97,106-171): the weights
// w = rmin - sqrt(dx^2+dy^2+dz^2) of the box are derived once per CTA into
// shared memory; neighbours are summed in the reference's order (dx outer,
// dz inner), skipping w <= 0 and out-of-domain elements.
//   density: out = sum w x_j / (sum w + 1e-20)
//   sens:    out = sum w rho_j dc_j / (rho_e sum w + 1e-20)
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(H3_FLAT)
    k_hex_filter(Hex3 g, double rmin, int R, const double *__restrict__ x,
                 const double *__restrict__ rho, double *__restrict__ out) {
  extern __shared__ double hw[];
  const int W = 2 * R + 1;
  for (int k = threadIdx.x; k < W * W * W; k += blockDim.x) {
    const int dx = k / (W * W) - R, dy = (k / W) % W - R, dz = k % W - R;
    hw[k] = rmin - sqrt((double)(dx * dx + dy * dy + dz * dz));
  }
  __syncthreads();
  const int64_t ne = g.elems();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = e / g.nz;
    const int ez = (int)(e - col * g.nz);
    const int ex = (int)(col / g.ny);
    const int ey = (int)(col - (int64_t)ex * g.ny);
    double num = 0.0, den = 0.0;
    for (int dx = -R; dx <= R; ++dx) {
      const int jx = ex + dx;
      if (jx < 0 || jx >= g.nx) continue;
      for (int dy = -R; dy <= R; ++dy) {
        const int jy = ey + dy;
        if (jy < 0 || jy >= g.ny) continue;
        const double *wrow = hw + ((dx + R) * W + (dy + R)) * W + R;
        const int64_t jbase = ((int64_t)jx * g.ny + jy) * g.nz;
        for (int dz = -R; dz <= R; ++dz) {
          const int jz = ez + dz;
          const double w = wrow[dz];
          if (w > 0.0 && jz >= 0 && jz < g.nz) {
            const int64_t j = jbase + jz;
            const double v = (MODE == F_SENS) ? rho[j] * x[j] : x[j];
            num = fma(w, v, num);
            den += w;
          }
        }
      }
    }
    out[e] = (MODE == F_SENS) ? num / (rho[e] * den + 1e-20) : num / (den + 1e-20);
  }
}

}  // namespace tpo
