// libtpo: host side of the 3D (H8) entry points, tpo3_* in include/tpo.h.
// Included at the end of api.cu (same translation unit: the error, launch
// and polling helpers and the __constant__ stiffness are shared).
#pragma once

namespace {

bool g_have_stiffness3[kMaxDevices];
double g_alpha_reg3[kMaxDevices];
bool g_h8_structured[kMaxDevices];  // Ke is lam K_lam + mu K_mu: k_hex_elem applies it

// Launch-size caps: grid-stride loops cover larger grids, and the grid
// reductions read at most this many partials.
constexpr int kHexMaxCtas = 2048;

int check_grid3(const tpo_grid3 *g) {
  if (!g) return fail(TPO_ERR_ARGS, "grid is NULL");
  if (g->nelx < 1 || g->nely < 1 || g->nelz < 1)
    return fail(TPO_ERR_ARGS, "nelx, nely, nelz must be >= 1");
  if ((int64_t)(g->nelx + 1) * (g->nely + 1) * (g->nelz + 1) > ((int64_t)1 << 30))
    return fail(TPO_ERR_ARGS, "grid too large");
  return TPO_OK;
}

int need_stiffness3(int *dev) {
  int rc = current_device(dev);
  if (rc) return rc;
  if (!g_have_stiffness3[*dev])
    return fail(TPO_ERR_NO_STIFFNESS, "tpo_set_stiffness3 has not been called on device %d",
                *dev);
  return TPO_OK;
}

Hex3 hex_of(const tpo_grid3 *g) { return Hex3{g->nelx, g->nely, g->nelz}; }
dim3 hex_gather_grid(const Hex3 &h) { return flat_grid(h.nodes(), H3_THREADS, kHexMaxCtas); }
dim3 hex_elem_grid(const Hex3 &h) { return flat_grid(h.elems(), H3_THREADS, kHexMaxCtas); }
dim3 hex_flat_grid(int64_t n) { return flat_grid(n, H3_FLAT, kHexMaxCtas); }

// CTAs of `kernel` resident per SM (1 if the query fails).
template <typename K>
int resident_ctas(K kernel, int threads, size_t smem) {
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess ||
      nb < 1) {
    cudaGetLastError();
    return 1;
  }
  return nb;
}

// Launch plan of the nodal gathers: the plane-marching kernel when its
// staging fits in shared memory (nelz up to ~700) and one x-plane takes at
// most kHexMaxCtas CTAs, the per-node kernel otherwise. The planes are split
// into chunks of xc consecutive planes so that the grid is one wave of
// resident CTAs (longer marches amortise the two-plane prologue).
constexpr size_t kTileSmemMax = 220 * 1024;
struct GatherPlan {
  bool tile = false;
  dim3 grid;
  int xc = 0;
  size_t smem = 0;
  // element-centric structured kernel (matvec, direction, residual)
  bool elem = false;
  dim3 egrid;
  int ey = 0, ez = 0, tzc = 0, exc = 0;
  size_t esmem = 0;
};

// Tiles of the element-centric kernel: EY x EZ elements (EY EZ <= HE_THREADS)
// finish (EY-1) x (EZ-1) nodes; the shape that needs the fewest element slots
// per plane to cover the (nely+1) x (nelz+1) nodes, then chunks of planes
// for about one wave of resident CTAs.
void elem_plan(const Hex3 &h, GatherPlan &p) {
  int dev = 0;
  if (current_device(&dev) || !g_h8_structured[dev]) return;
  int64_t best = -1;
  for (int ez = 3; ez <= HE_THREADS / 3; ++ez) {
    const int ey = HE_THREADS / ez;
    const int64_t tzc = (h.nz + 1 + ez - 2) / (ez - 1), tyc = (h.ny + 1 + ey - 2) / (ey - 1);
    const int64_t cost = tzc * tyc * ey * ez;
    if (tzc * tyc > kHexMaxCtas || hex_elem_smem(ey, ez) > kTileSmemMax ||
        3 * hex_elem_ns(ey, ez) > HE_KS * HE_THREADS)
      continue;
    if (best < 0 || cost < best) {
      best = cost;
      p.ey = ey;
      p.ez = ez;
      p.tzc = (int)tzc;
    }
  }
  if (best < 0) return;
  const int64_t tiles = (int64_t)p.tzc * ((h.ny + 1 + p.ey - 2) / (p.ey - 1));
  p.esmem = hex_elem_smem(p.ey, p.ez);
  const int64_t planes = (int64_t)h.nx + 1;
  const int64_t wave =
      (int64_t)resident_ctas(k_hex_elem<H3_DIR, 0>, HE_THREADS, p.esmem) * sm_count();
  int64_t chunks = std::max<int64_t>(1, wave / tiles);
  chunks = std::min<int64_t>(std::min<int64_t>(chunks, planes), kHexMaxCtas / tiles);
  const int64_t xc = (planes + chunks - 1) / chunks;
  chunks = (planes + xc - 1) / xc;
  p.egrid = dim3((unsigned)tiles, (unsigned)chunks, 1);
  p.exc = (int)xc;
  p.elem = true;
}

GatherPlan gather_plan(const Hex3 &h) {
  GatherPlan p;
  const int64_t P = (int64_t)(h.ny + 1) * (h.nz + 1);
  const int64_t cpp = (P + HT_THREADS - 1) / HT_THREADS;
  const size_t smem = hex_tile_smem(h.nz);
  elem_plan(h, p);
  if (smem > kTileSmemMax || cpp > kHexMaxCtas) {
    p.grid = hex_gather_grid(h);
    return p;
  }
  const int64_t planes = (int64_t)h.nx + 1;
  const int64_t wave = (int64_t)resident_ctas(k_hex_tile<H3_DIR, 0>, HT_THREADS, smem) * sm_count();
  int64_t chunks = std::max<int64_t>(1, wave / cpp);
  chunks = std::min<int64_t>(std::min<int64_t>(chunks, planes), kHexMaxCtas / cpp);
  const int64_t xc = (planes + chunks - 1) / chunks;
  chunks = (planes + xc - 1) / xc;
  p.tile = true;
  p.grid = dim3((unsigned)cpp, (unsigned)chunks, 1);
  p.xc = (int)xc;
  p.smem = smem;
  return p;
}

template <int MODE, int PRE>
int launch_gather(const GatherPlan &p, const Hex3Args &a, cudaStream_t st) {
  if constexpr (MODE != H3_BLOCK) {
    if (p.elem) {
      if (p.esmem > 48 * 1024)
        TPO_CK(cudaFuncSetAttribute(k_hex_elem<MODE, PRE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.esmem));
      k_hex_elem<MODE, PRE><<<p.egrid, HE_THREADS, p.esmem, st>>>(a, p.ey, p.ez, p.tzc, p.exc);
      TPO_CK_LAUNCH();
      return TPO_OK;
    }
  }
  if (p.tile) {
    if (p.smem > 48 * 1024)
      TPO_CK(cudaFuncSetAttribute(k_hex_tile<MODE, PRE>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem));
    k_hex_tile<MODE, PRE><<<p.grid, HT_THREADS, p.smem, st>>>(a, p.xc);
  } else {
    k_hex_gather<MODE, PRE><<<p.grid, H3_THREADS, 0, st>>>(a);
  }
  TPO_CK_LAUNCH();
  return TPO_OK;
}

struct Pcg3Ws {
  PcgCtl *ctl;
  double *s, *w, *diag, *r, *z, *pa, *pb, *ap, *part;
  size_t bytes;
};

Pcg3Ws carve_pcg3(void *base, const tpo_grid3 *g, const tpo_solve_cfg *c) {
  const Hex3 h = hex_of(g);
  const size_t ne = h.elems(), nd = 3 * h.nodes();
  Carve cv(base);
  Pcg3Ws w{};
  w.ctl = cv.take<PcgCtl>(1);
  w.s = cv.take<double>(ne);
  if (c->precond == TPO_PRECOND_BLOCK_JACOBI) w.w = cv.take<double>(ne);
  if (c->precond == TPO_PRECOND_JACOBI) w.diag = cv.take<double>(nd);
  w.r = cv.take<double>(nd);
  if (c->precond != TPO_PRECOND_NONE) w.z = cv.take<double>(nd);
  w.pa = cv.take<double>(nd);
  w.pb = cv.take<double>(nd);
  w.ap = cv.take<double>(nd);
  w.part = cv.take<double>(2 * (size_t)kHexMaxCtas);
  w.bytes = cv.off;
  return w;
}

template <int PRE>
int pcg3(const tpo_grid3 *g, const tpo_solve_cfg *c, const double *rho, const double *f,
         const uint8_t *fixed, double *u, const Pcg3Ws &w, tpo_solve_result *out,
         cudaStream_t st, double alpha_reg) {
  const Hex3 h = hex_of(g);
  const int64_t nn = h.nodes(), nd = 3 * nn, ne = h.elems();
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);
  const dim3 gg = hex_gather_grid(h);
  const GatherPlan gp = gather_plan(h);
  // the update streams 8 vectors: one wave of resident CTAs, grid-stride;
  // 16-byte accesses when every array allows them
  const bool vec = aligned(u, 16) && aligned(w.r, 16) && aligned(w.pa, 16) &&
                   aligned(w.pb, 16) && aligned(w.ap, 16) && aligned(w.diag, 16) &&
                   aligned(w.z, 16);
  const dim3 fg = flat_grid(nd, H3_FLAT,
                            std::min(kHexMaxCtas, resident_ctas(k_hex_update<PRE>, H3_FLAT, 0) *
                                                      sm_count()));
  const dim3 fg2 = flat_grid(nd / 2 + 1, H3_FLAT,
                             std::min(kHexMaxCtas, resident_ctas(k_hex_update2<PRE>, H3_FLAT, 0) *
                                                       sm_count()));
  // warm start from u with its fixed DOFs zeroed, else from zero (solver.py:52-57)
  if (c->warm_start) {
    k_hex_zero_fixed<<<hex_flat_grid(nn), H3_FLAT, 0, st>>>(nn, fixed, u);
    TPO_CK_LAUNCH();
  } else {
    TPO_CK(cudaMemsetAsync(u, 0, nd * sizeof(double), st));
  }
  k_hex_scales<<<hex_flat_grid(ne), H3_FLAT, 0, st>>>(ne, rho, g->e_min, g->penalty, alpha_reg,
                                                      w.s, w.w);
  TPO_CK_LAUNCH();
  if (PRE == TPO_PRECOND_JACOBI) {
    k_hex_diag<<<gg, H3_THREADS, 0, st>>>(h, w.s, fixed, w.diag);
    TPO_CK_LAUNCH();
  }
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, 0.0, c->max_iter, nullptr, 0.0, 0);
  TPO_CK_LAUNCH();

  Hex3Args a{};
  a.g = h;
  a.w = w.s;
  a.mask = fixed;
  a.part = w.part;
  a.ctl = w.ctl;
  // r = f - K u, z = M r (point preconditioners), r.z, ||r||^2
  a.x = u;
  a.f = f;
  a.diag = w.diag;
  a.out = w.r;
  a.z = w.z;
  int rc = launch_gather<H3_RES, PRE>(gp, a, st);
  if (rc) return rc;
  Hex3Args b{};  // element-block z = M r
  b.g = h;
  b.w = w.w;
  b.mask = fixed;
  b.x = w.r;
  b.out = w.z;
  b.part = w.part;
  b.ctl = w.ctl;
  if (PRE == TPO_PRECOND_BLOCK_JACOBI) {
    b.init = 1;
    if ((rc = launch_gather<H3_BLOCK, 0>(gp, b, st))) return rc;
    b.init = 0;
  }
  Hex3Args d{};  // p' = z + beta p, ap = K p', alpha
  d.g = h;
  d.w = w.s;
  d.mask = fixed;
  d.x = PRE == TPO_PRECOND_NONE ? w.r : w.z;
  d.pa = w.pa;
  d.pb = w.pb;
  d.out = w.ap;
  d.part = w.part;
  d.ctl = w.ctl;

  auto iter = [&](cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    int r = launch_gather<H3_DIR, 0>(gp, d, st);
    if (r) return r;
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    if (ev) TPO_CK(cudaEventRecord(ev[2], st));
    if (vec)
      k_hex_update2<PRE><<<fg2, H3_FLAT, 0, st>>>(nd, u, w.r, w.pa, w.pb, w.ap, w.diag, w.z,
                                                  w.part, w.ctl);
    else
      k_hex_update<PRE><<<fg, H3_FLAT, 0, st>>>(nd, u, w.r, w.pa, w.pb, w.ap, w.diag, w.z,
                                                w.part, w.ctl);
    TPO_CK_LAUNCH();
    if (PRE == TPO_PRECOND_BLOCK_JACOBI && (r = launch_gather<H3_BLOCK, 0>(gp, b, st))) return r;
    if (ev) TPO_CK(cudaEventRecord(ev[3], st));
    return TPO_OK;
  };
  // algorithmic bytes: direction z|r, p_old -> p', ap; scales; mask. Update:
  // u, r, p', ap -> u, r (+ diag -> z); element-block: r -> z, weights, mask.
  LaunchBytes lb{};
  lb.dir = 4 * nd * 8 + ne * 8 + nn;
  lb.update = 6 * nd * 8 + (PRE == TPO_PRECOND_JACOBI ? 2 * nd * 8 : 0) +
              (PRE == TPO_PRECOND_BLOCK_JACOBI ? 2 * nd * 8 + ne * 8 + nn : 0);
  PcgCtl fin;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  rc = run_iterations(iter, w.ctl, c->max_iter, 0, chunk, st, &fin, lb);
  if (rc) return rc;
  int status = fin.status;
  if (status == TPO_SOLVE_RUNNING) status = TPO_SOLVE_MAX_ITER;  // max_iter <= 0
  out->status = status;
  out->updates = fin.it;
  out->iters = (status == TPO_SOLVE_CONVERGED) ? fin.it : c->max_iter;
  out->outer_iters = 1;
  out->rr = fin.rr;
  return TPO_OK;
}

struct Sens3Ws {
  SumCtl *ctl;
  double *part;
  size_t bytes;
};
Sens3Ws carve_sens3(void *base) {
  Carve cv(base);
  Sens3Ws w{};
  w.ctl = cv.take<SumCtl>(1);
  w.part = cv.take<double>(2 * (size_t)kHexMaxCtas);
  w.bytes = cv.off;
  return w;
}

int filter3_launch(const tpo_grid3 *g, double rmin, int mode, const double *x, const double *rho,
                   double *out, tpo_stream s) {
  int rc = check_grid3(g);
  if (rc) return rc;
  if (!x || !out || (mode == F_SENS && !rho)) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!(rmin > 0.0)) return fail(TPO_ERR_ARGS, "rmin must be > 0");
  const int R = (int)std::ceil(rmin);
  if (R > H3_MAXR) return fail(TPO_ERR_ARGS, "ceil(rmin) = %d > %d", R, H3_MAXR);
  const int W = 2 * R + 1;
  const size_t smem = (size_t)W * W * W * sizeof(double);
  const Hex3 h = hex_of(g);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  const dim3 gr = hex_flat_grid(h.elems());
  if (mode == F_SENS)
    k_hex_filter<F_SENS><<<gr, H3_FLAT, smem, st>>>(h, rmin, R, x, rho, out);
  else
    k_hex_filter<F_DENSITY><<<gr, H3_FLAT, smem, st>>>(h, rmin, R, x, nullptr, out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// The OC bisection is pointwise over elements: the 3D design runs through the
// same kernels as a 2D grid of E x 1 elements.
tpo_grid flat_oc_grid(const tpo_grid3 *g) {
  tpo_grid f{};
  f.nelx = (int32_t)hex_of(g).elems();
  f.nely = 1;
  f.e_min = g->e_min;
  f.penalty = g->penalty;
  return f;
}

// Ke as lam K_lam + mu K_mu, the unit-cube isotropic H8 operator
// (h8_forces): least squares over the 576 entries, accepted when every entry
// agrees to 1e-12 of the largest. Otherwise the dense gathers apply Ke.
bool h8_fit(const double ke[576], double *lam, double *mu) {
  static const int dxyz[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};  // reference order
  int bit_of[8];
  for (int r = 0; r < 8; ++r) bit_of[r] = dxyz[r][0] + 2 * dxyz[r][1] + 4 * dxyz[r][2];
  std::vector<double> kl(576), km(576);
  const H8Const cl = h8_const(1.0, 0.0), cm = h8_const(0.0, 1.0);
  for (int col = 0; col < 24; ++col) {
    double v[8][3] = {}, fl[8][3], fm[8][3];
    v[bit_of[col / 3]][col % 3] = 1.0;
    h8_forces(cl, 1.0, v, fl);
    h8_forces(cm, 1.0, v, fm);
    for (int row = 0; row < 24; ++row) {
      kl[row * 24 + col] = fl[bit_of[row / 3]][row % 3];
      km[row * 24 + col] = fm[bit_of[row / 3]][row % 3];
    }
  }
  double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0, kmax = 0;
  for (int i = 0; i < 576; ++i) {
    a11 += kl[i] * kl[i];
    a12 += kl[i] * km[i];
    a22 += km[i] * km[i];
    b1 += kl[i] * ke[i];
    b2 += km[i] * ke[i];
    kmax = std::max(kmax, std::fabs(ke[i]));
  }
  const double det = a11 * a22 - a12 * a12;
  if (!(det > 0.0) || !(kmax > 0.0)) return false;
  *lam = (b1 * a22 - b2 * a12) / det;
  *mu = (a11 * b2 - a12 * b1) / det;
  for (int i = 0; i < 576; ++i)
    if (std::fabs(ke[i] - (*lam * kl[i] + *mu * km[i])) > 1e-12 * kmax) return false;
  return true;
}

}  // namespace

extern "C" {

int tpo_set_stiffness3(const double ke[576], const double ke_inv[576], double alpha_reg) {
  if (!ke || !ke_inv) return fail(TPO_ERR_ARGS, "ke and ke_inv must be non-NULL");
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  for (int i = 0; i < 576; ++i)
    if (!std::isfinite(ke[i]) || !std::isfinite(ke_inv[i]))
      return fail(TPO_ERR_ARGS, "non-finite stiffness entry %d", i);
  TPO_CK(cudaMemcpyToSymbol(c_ke3, ke, sizeof(double) * 576));
  TPO_CK(cudaMemcpyToSymbol(c_kinv3, ke_inv, sizeof(double) * 576));
  double lam = 0.0, mu = 0.0;
  g_h8_structured[dev] = h8_fit(ke, &lam, &mu);
  if (g_h8_structured[dev]) {
    const H8Const k = h8_const(lam, mu);
    TPO_CK(cudaMemcpyToSymbol(c_h8s, &k, sizeof(H8Const)));
  }
  g_alpha_reg3[dev] = alpha_reg;
  g_have_stiffness3[dev] = true;
  return TPO_OK;
}

size_t tpo3_matvec_workspace_bytes(const tpo_grid3 *g) {
  if (check_grid3(g)) return 0;
  Carve cv(nullptr);
  cv.take<SumCtl>(1);
  cv.take<double>(2 * (size_t)kHexMaxCtas);
  cv.take<double>((size_t)hex_of(g).elems());
  return cv.off;
}

int tpo3_matvec_f64(const tpo_grid3 *g, const double *rho, const uint8_t *fixed, const double *p,
                    double *ap, double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid3(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness3(&dev))) return rc;
  if (!rho || !fixed || !p || !ap || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(p, 8) || !aligned(ap, 8) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer");
  if (ws_bytes < tpo3_matvec_workspace_bytes(g))
    return fail(TPO_ERR_WORKSPACE, "workspace too small");
  const Hex3 h = hex_of(g);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  Carve cv(ws);
  SumCtl *ctl = cv.take<SumCtl>(1);
  double *part = cv.take<double>(2 * (size_t)kHexMaxCtas);
  double *sc = cv.take<double>((size_t)h.elems());
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(SumCtl), st));
  k_hex_scales<<<hex_flat_grid(h.elems()), H3_FLAT, 0, st>>>(h.elems(), rho, g->e_min,
                                                             g->penalty, 0.0, sc, nullptr);
  TPO_CK_LAUNCH();
  Hex3Args a{};
  a.g = h;
  a.w = sc;
  a.mask = fixed;
  a.x = p;
  a.out = ap;
  a.part = part;
  a.counter = &ctl->counter;
  a.pap_out = pap_out;
  cudaEvent_t *ev = nullptr;
  if (g_prof_on && (rc = prof_events(1, &ev))) return rc;
  if (ev) TPO_CK(cudaEventRecord(ev[0], st));
  if ((rc = launch_gather<H3_APPLY, 0>(gather_plan(h), a, st))) return rc;
  if (ev) {
    TPO_CK(cudaEventRecord(ev[1], st));
    TPO_CK(cudaEventSynchronize(ev[1]));
    float ms = 0.f;
    TPO_CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    g_prof.apply_launches += 1;
    g_prof.apply_ms += ms;
    g_prof.apply_bytes += 2 * 3 * h.nodes() * 8 + h.elems() * 8 + h.nodes();
  }
  return TPO_OK;
}

size_t tpo3_pcg_workspace_bytes(const tpo_grid3 *g, const tpo_solve_cfg *c) {
  if (check_grid3(g) || !c) return 0;
  return carve_pcg3(nullptr, g, c).bytes;
}

int tpo3_pcg_solve(const tpo_grid3 *g, const tpo_solve_cfg *c, const double *rho_phys,
                   const double *f, const uint8_t *fixed, double *u, void *ws, size_t ws_bytes,
                   tpo_solve_result *out, tpo_stream s) {
  int rc = check_grid3(g);
  if (rc) return rc;
  if (!c || !out) return fail(TPO_ERR_ARGS, "cfg and result must be non-NULL");
  int dev;
  if ((rc = need_stiffness3(&dev))) return rc;
  if (!rho_phys || !f || !fixed || !u || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(f, 8) || !aligned(u, 8) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer (vectors need 8 B, workspace 256 B)");
  if (c->precond != TPO_PRECOND_NONE && c->precond != TPO_PRECOND_JACOBI &&
      c->precond != TPO_PRECOND_BLOCK_JACOBI)
    return fail(TPO_ERR_ARGS, "3D solves take none, jacobi or block_jacobi (got %d)", c->precond);
  if (c->precision != TPO_PRECISION_FP64)
    return fail(TPO_ERR_ARGS, "3D solves are FP64 only");
  if (c->recurrence != TPO_RECURRENCE_AUTO && c->recurrence != TPO_RECURRENCE_STANDARD)
    return fail(TPO_ERR_ARGS, "3D solves use the standard recurrence");
  if (!(c->tol >= 0.0) || !(c->f_norm_sq >= 0.0))
    return fail(TPO_ERR_ARGS, "tol and f_norm_sq must be >= 0");
  const Pcg3Ws w = carve_pcg3(ws, g, c);
  if (ws_bytes < w.bytes) return fail(TPO_ERR_WORKSPACE, "workspace %zu < %zu", ws_bytes, w.bytes);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  memset(out, 0, sizeof(*out));
  if (std::sqrt(c->f_norm_sq) < 1e-30) {  // reference solver.py:59-63
    TPO_CK(cudaMemsetAsync(u, 0, 3 * hex_of(g).nodes() * sizeof(double), st));
    TPO_CK(cudaStreamSynchronize(st));
    out->status = TPO_SOLVE_ZERO_RHS;
    return TPO_OK;
  }
  const double ar = g_alpha_reg3[dev];
  switch (c->precond) {
    case TPO_PRECOND_NONE:
      return pcg3<TPO_PRECOND_NONE>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    case TPO_PRECOND_JACOBI:
      return pcg3<TPO_PRECOND_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    default:
      return pcg3<TPO_PRECOND_BLOCK_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
  }
}

size_t tpo3_sensitivity_workspace_bytes(const tpo_grid3 *g) {
  if (check_grid3(g)) return 0;
  return carve_sens3(nullptr).bytes;
}

int tpo3_sensitivity(const tpo_grid3 *g, const double *rho_phys, const double *u, double *dc,
                     double *compliance_out, void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid3(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness3(&dev))) return rc;
  if (!rho_phys || !u || !dc || !compliance_out || !ws)
    return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(ws, kAlign)) return fail(TPO_ERR_ARGS, "misaligned workspace");
  const Sens3Ws w = carve_sens3(ws);
  if (ws_bytes < w.bytes) return fail(TPO_ERR_WORKSPACE, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  TPO_CK(cudaMemsetAsync(w.ctl, 0, sizeof(SumCtl), st));
  const Hex3 h = hex_of(g);
  k_hex_sensitivity<<<hex_elem_grid(h), H3_THREADS, 0, st>>>(h, g->e_min, g->penalty, rho_phys,
                                                            u, dc, w.part, w.ctl, compliance_out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

int tpo3_density_filter(const tpo_grid3 *g, double rmin, const double *x, double *out,
                        tpo_stream s) {
  return filter3_launch(g, rmin, F_DENSITY, x, nullptr, out, s);
}

int tpo3_sensitivity_filter(const tpo_grid3 *g, double rmin, const double *rho, const double *dc,
                            double *out, tpo_stream s) {
  return filter3_launch(g, rmin, F_SENS, dc, rho, out, s);
}

size_t tpo3_oc_workspace_bytes(const tpo_grid3 *g) {
  if (check_grid3(g)) return 0;
  const tpo_grid f = flat_oc_grid(g);
  return tpo_oc_workspace_bytes(&f);
}

int tpo3_oc_update(const tpo_grid3 *g, double volfrac, double move, const double *rho_in,
                   const double *dc, const double *dv, double *rho_out, double *result_out,
                   void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid3(g);
  if (rc) return rc;
  const tpo_grid f = flat_oc_grid(g);
  return tpo_oc_update(&f, volfrac, move, rho_in, dc, dv, rho_out, result_out, ws, ws_bytes, s);
}

}  // extern "C"
