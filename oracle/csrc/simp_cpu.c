/*
 * simp_cpu.c -- C/OpenMP restatement of the reference's SIMP loop, FP64,
 * on 2D (Q4) and 3D (H8) structured grids.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY: used by tests/ as a fast oracle and
 * by bench.py as the timed CPU baseline (the reference's own CPU path runs on
 * Taichi, which this image cannot install). Never linked into libtpo.
 *
 * It follows the reference algorithm kernel by kernel, in the reference's
 * element-scatter form (tomohiron907/toptimization, src/toptimization/):
 *   matvec        fem/kernels.py:143-212   (element scatter in 4 (2D) or 8
 *                                           (3D) parity colours, so the
 *                                           parallel scatter needs no atomics)
 *   jacobi diag   fem/kernels.py:76-129
 *   element block fem/preconditioner.py:19-156, fem/fields.py:133-143
 *   PCG           fem/solver.py:27-159
 *   sensitivity   fem/kernels.py:234-308
 *   filters       optimizer/filter.py:22-171 (weights recomputed per box)
 *   OC            optimizer/oc.py:21-93
 *   SIMP loop     optimizer/simp.py:141-219
 * plus the 2x2 nodal block-Jacobi option (2D only), which has no reference
 * counterpart. 3D numbering (mesh.py:68-112): node (ix*(ny+1)+iy)*(nz+1)+iz,
 * element (ex*ny+ey)*nz+ez, H8 corners bottom face then top face.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { PC_NONE = 0, PC_JACOBI = 1, PC_BLOCK = 2, PC_NODAL = 3 };

typedef struct {
  int nx, ny, nz, dim, dpe, precond, max_cg, filter_sens; /* nz = 0: 2D */
  double e_min, pen, rmin, volfrac, move, cg_tol, alpha_reg, f_norm;
  size_t nn, ndof, ne;
  double *ke, *kinv; /* dpe x dpe */
  double *f, *u, *r, *p, *ap, *z, *diag, *scale, *w;
  double *rho, *rho_phys, *dc, *dc_filt, *tmp, *binv; /* binv: 3 per node */
  uint8_t *fixed; /* per DOF */
  int it;
} ocpu;

/* DOFs of element (ex, ey, ez) in the reference's order (ez = 0 in 2D) */
static inline void elem_dofs(const ocpu *c, int ex, int ey, int ez, long d[24]) {
  const long ny1 = c->ny + 1;
  if (c->dim == 2) {
    const long n1 = ex * ny1 + ey, n2 = (ex + 1) * ny1 + ey, n3 = n2 + 1, n4 = n1 + 1;
    d[0] = 2 * n1; d[1] = 2 * n1 + 1; d[2] = 2 * n2; d[3] = 2 * n2 + 1;
    d[4] = 2 * n3; d[5] = 2 * n3 + 1; d[6] = 2 * n4; d[7] = 2 * n4 + 1;
    return;
  }
  static const int cx[8] = {0, 1, 1, 0, 0, 1, 1, 0}, cy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                   cz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  const long nz1 = c->nz + 1;
  for (int k = 0; k < 8; ++k) {
    const long n = ((long)(ex + cx[k]) * ny1 + ey + cy[k]) * nz1 + ez + cz[k];
    d[3 * k] = 3 * n; d[3 * k + 1] = 3 * n + 1; d[3 * k + 2] = 3 * n + 2;
  }
}

static inline long elem_index(const ocpu *c, int ex, int ey, int ez) {
  return c->dim == 2 ? (long)ex * c->ny + ey : ((long)ex * c->ny + ey) * c->nz + ez;
}
static inline void elem_coords(const ocpu *c, long e, int *ex, int *ey, int *ez) {
  if (c->dim == 2) {
    *ex = (int)(e / c->ny); *ey = (int)(e % c->ny); *ez = 0;
  } else {
    *ez = (int)(e % c->nz); *ey = (int)((e / c->nz) % c->ny); *ex = (int)(e / ((long)c->nz * c->ny));
  }
}
static inline int ncolors(const ocpu *c) { return c->dim == 2 ? 4 : 8; }

static double dot(const double *a, const double *b, size_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < (long)n; ++i) s += a[i] * b[i];
  return s;
}

/* out = sum_e s_e M p_e (element scatter in parity colours: elements of one
 * colour share no node), M = Ke or Ke_inv. */
static void scatter_apply(const ocpu *c, const double *m, const double *s, const double *in,
                          double *out) {
  memset(out, 0, c->ndof * sizeof(double));
  const int dpe = c->dpe, nzl = c->dim == 2 ? 1 : c->nz;
  for (int color = 0; color < ncolors(c); ++color) {
    const int cx = color & 1, cy = (color >> 1) & 1, cz = color >> 2;
#pragma omp parallel for schedule(static)
    for (int ex = cx; ex < c->nx; ex += 2) {
      for (int ey = cy; ey < c->ny; ey += 2) {
        for (int ez = cz; ez < nzl; ez += 2) {
          long d[24];
          elem_dofs(c, ex, ey, ez, d);
          const double se = s[elem_index(c, ex, ey, ez)];
          double pl[24];
          for (int j = 0; j < dpe; ++j) pl[j] = in[d[j]];
          for (int i = 0; i < dpe; ++i) {
            double acc = 0.0;
            for (int j = 0; j < dpe; ++j) acc += m[i * dpe + j] * pl[j];
            out[d[i]] += se * acc;
          }
        }
      }
    }
  }
}

static void matvec(const ocpu *c, const double *p, double *ap) {
  scatter_apply(c, c->ke, c->scale, p, ap);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)c->ndof; ++i)
    if (c->fixed[i]) ap[i] = p[i];
}

static void setup_precond(ocpu *c) {
  if (c->precond == PC_JACOBI) {
    const int dpe = c->dpe, nzl = c->dim == 2 ? 1 : c->nz;
    memset(c->diag, 0, c->ndof * sizeof(double));
    for (int color = 0; color < ncolors(c); ++color) {
      const int cx = color & 1, cy = (color >> 1) & 1, cz = color >> 2;
#pragma omp parallel for schedule(static)
      for (int ex = cx; ex < c->nx; ex += 2)
        for (int ey = cy; ey < c->ny; ey += 2)
          for (int ez = cz; ez < nzl; ez += 2) {
            long d[24];
            elem_dofs(c, ex, ey, ez, d);
            const double se = c->scale[elem_index(c, ex, ey, ez)];
            for (int i = 0; i < dpe; ++i) c->diag[d[i]] += se * c->ke[i * (dpe + 1)];
          }
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)c->ndof; ++i) {
      if (c->fixed[i]) c->diag[i] = 1.0;
      else if (c->diag[i] < 1e-20) c->diag[i] = 1e-20;
    }
  } else if (c->precond == PC_BLOCK) {
#pragma omp parallel for schedule(static)
    for (long e = 0; e < (long)c->ne; ++e) {
      const double s = c->scale[e], sc = s > c->alpha_reg ? s : c->alpha_reg;
      c->w[e] = s / (sc * sc);
    }
    /* diag holds 1/sqrt(count) per DOF: elements sharing the node */
#pragma omp parallel for schedule(static)
    for (long n = 0; n < (long)c->nn; ++n) {
      int x, y, z = 0;
      if (c->dim == 2) {
        x = (int)(n / (c->ny + 1)); y = (int)(n % (c->ny + 1));
      } else {
        z = (int)(n % (c->nz + 1)); y = (int)((n / (c->nz + 1)) % (c->ny + 1));
        x = (int)(n / ((long)(c->nz + 1) * (c->ny + 1)));
      }
      int cnt = ((x >= 1) + (x <= c->nx - 1)) * ((y >= 1) + (y <= c->ny - 1));
      if (c->dim == 3) cnt *= (z >= 1) + (z <= c->nz - 1);
      for (int k = 0; k < c->dim; ++k) c->diag[c->dim * n + k] = 1.0 / sqrt((double)cnt);
    }
  } else if (c->precond == PC_NODAL) {
    double *b = c->tmp; /* 3 per node, nn <= ne + ... : use binv as scratch */
    (void)b;
    memset(c->binv, 0, 3 * c->nn * sizeof(double));
    for (int color = 0; color < 4; ++color) {
      const int cx = color & 1, cy = color >> 1;
#pragma omp parallel for schedule(static)
      for (int ex = cx; ex < c->nx; ex += 2)
        for (int ey = cy; ey < c->ny; ey += 2) {
          long d[24];
          elem_dofs(c, ex, ey, 0, d);
          const double se = c->scale[(long)ex * c->ny + ey];
          for (int a = 0; a < 4; ++a) {
            const long n = d[2 * a] / 2;
            c->binv[3 * n + 0] += se * c->ke[(2 * a) * 8 + 2 * a];
            c->binv[3 * n + 1] += se * c->ke[(2 * a) * 8 + 2 * a + 1];
            c->binv[3 * n + 2] += se * c->ke[(2 * a + 1) * 8 + 2 * a + 1];
          }
        }
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < (long)c->nn; ++n) {
      double bxx = c->binv[3 * n], bxy = c->binv[3 * n + 1], byy = c->binv[3 * n + 2];
      if (c->fixed[2 * n]) { bxx = 1.0; bxy = 0.0; }
      if (c->fixed[2 * n + 1]) { byy = 1.0; bxy = 0.0; }
      const double det = bxx * byy - bxy * bxy;
      c->binv[3 * n] = byy / det;
      c->binv[3 * n + 1] = -bxy / det;
      c->binv[3 * n + 2] = bxx / det;
    }
  }
}

static void apply_precond(const ocpu *c, const double *r, double *z) {
  if (c->precond == PC_JACOBI) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)c->ndof; ++i) z[i] = r[i] / c->diag[i];
  } else if (c->precond == PC_BLOCK) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)c->ndof; ++i) c->tmp[i] = r[i] * c->diag[i];
    scatter_apply(c, c->kinv, c->w, c->tmp, z);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)c->ndof; ++i) z[i] = c->fixed[i] ? 0.0 : z[i] * c->diag[i];
  } else if (c->precond == PC_NODAL) {
#pragma omp parallel for schedule(static)
    for (long n = 0; n < (long)c->nn; ++n) {
      const double rx = r[2 * n], ry = r[2 * n + 1];
      z[2 * n] = c->binv[3 * n] * rx + c->binv[3 * n + 1] * ry;
      z[2 * n + 1] = c->binv[3 * n + 1] * rx + c->binv[3 * n + 2] * ry;
    }
  } else {
    memcpy(z, r, c->ndof * sizeof(double));
  }
}

/* reference fem/solver.py:27-159; returns the reference's count */
static int pcg(ocpu *c, int warm, int *status_out) {
  const size_t n = c->ndof;
  if (c->f_norm < 1e-30) {
    memset(c->u, 0, n * sizeof(double));
    *status_out = 5;
    return 0;
  }
  const double tol_sq = (c->cg_tol * c->f_norm) * (c->cg_tol * c->f_norm);
  setup_precond(c);
  if (!warm) memset(c->u, 0, n * sizeof(double));
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i)
    if (c->fixed[i]) c->u[i] = 0.0;
  matvec(c, c->u, c->ap);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) c->r[i] = c->f[i] - c->ap[i];
  apply_precond(c, c->r, c->z);
  memcpy(c->p, c->z, n * sizeof(double));
  double rz_old = dot(c->r, c->z, n);
  for (int it = 0; it < c->max_cg; ++it) {
    matvec(c, c->p, c->ap);
    const double pap = dot(c->p, c->ap, n);
    if (fabs(pap) < 1e-30) { *status_out = 3; return c->max_cg; }
    const double alpha = rz_old / pap;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
      c->u[i] += alpha * c->p[i];
      c->r[i] -= alpha * c->ap[i];
    }
    apply_precond(c, c->r, c->z);
    const double rz_new = dot(c->r, c->z, n);
    const double rr = dot(c->r, c->r, n);
    if (rr < tol_sq) { *status_out = 1; return it + 1; }
    const double beta = rz_new / (rz_old + 1e-60);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) c->p[i] = c->z[i] + beta * c->p[i];
    rz_old = rz_new;
  }
  *status_out = 2;
  return c->max_cg;
}

/* hat filter over the in-domain box, reference neighbour order */
static void hat_filter(const ocpu *c, const double *x, const double *rho, double *out, int sens) {
  const int R = (int)ceil(c->rmin);
  const int Rz = c->dim == 2 ? 0 : R, nzl = c->dim == 2 ? 1 : c->nz;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < (long)c->ne; ++e) {
    int ex, ey, ez;
    elem_coords(c, e, &ex, &ey, &ez);
    double num = 0.0, den = 0.0;
    for (int jx = ex - R; jx <= ex + R; ++jx) {
      if (jx < 0 || jx >= c->nx) continue;
      for (int jy = ey - R; jy <= ey + R; ++jy) {
        if (jy < 0 || jy >= c->ny) continue;
        for (int jz = ez - Rz; jz <= ez + Rz; ++jz) {
          if (jz < 0 || jz >= nzl) continue;
          const double dx = ex - jx, dy = ey - jy, dz = ez - jz;
          const double w = c->rmin - sqrt(dx * dx + dy * dy + dz * dz);
          if (w > 0.0) {
            const long j = elem_index(c, jx, jy, jz);
            num += sens ? w * rho[j] * x[j] : w * x[j];
            den += w;
          }
        }
      }
    }
    out[e] = sens ? num / (rho[e] * den + 1e-20) : num / (den + 1e-20);
  }
}

static double sensitivity(const ocpu *c, const double *rho) {
  double comp = 0.0;
#pragma omp parallel for reduction(+ : comp) schedule(static)
  for (long e = 0; e < (long)c->ne; ++e) {
    int ex, ey, ez;
    elem_coords(c, e, &ex, &ey, &ez);
    long d[24];
    elem_dofs(c, ex, ey, ez, d);
    const int dpe = c->dpe;
    double ul[24], uku = 0.0;
    for (int j = 0; j < dpe; ++j) ul[j] = c->u[d[j]];
    for (int i = 0; i < dpe; ++i) {
      double ku = 0.0;
      for (int j = 0; j < dpe; ++j) ku += c->ke[i * dpe + j] * ul[j];
      uku += ul[i] * ku;
    }
    const double r = rho[e];
    c->dc[e] = -c->pen * pow(r, c->pen - 1.0) * (1.0 - c->e_min) * uku;
    comp += (c->e_min + pow(r, c->pen) * (1.0 - c->e_min)) * uku;
  }
  return comp;
}

static double oc_update(ocpu *c, double *vol_out) {
  double lo = 0.0, hi = 1e9, change = 0.0, vol = 0.0, mid = 0.0;
  for (int k = 0; k < 50; ++k) {
    mid = 0.5 * (lo + hi);
    double vs = 0.0, ch = 0.0;
#pragma omp parallel for reduction(+ : vs) reduction(max : ch) schedule(static)
    for (long e = 0; e < (long)c->ne; ++e) {
      const double r = c->rho[e];
      double be = -c->dc_filt[e] / (mid + 1e-20);
      if (be < 0.0) be = 0.0;
      const double cand = r * sqrt(be);
      const double l = r - c->move > 0.001 ? r - c->move : 0.001;
      const double h = r + c->move < 1.0 ? r + c->move : 1.0;
      const double nw = cand < l ? l : (cand > h ? h : cand);
      c->tmp[e] = nw;
      vs += nw;
      const double d = fabs(nw - r);
      if (d > ch) ch = d;
    }
    change = ch;
    vol = vs / (double)c->ne;
    if (vol > c->volfrac) lo = mid; else hi = mid;
    if ((hi - lo) / (hi + lo + 1e-30) < 1e-4) break;
  }
  memcpy(c->rho, c->tmp, c->ne * sizeof(double));
  *vol_out = vol;
  return change;
}

/* ------------------------------------------------------------------ API */
/* nz = 0: 2D (ke, kinv 8x8); nz >= 1: 3D (ke, kinv 24x24). The nodal block
 * preconditioner is 2D only (NULL for 3D). */
void *ocpu_create(int nx, int ny, int nz, const double *ke, const double *kinv,
                  double alpha_reg, const int64_t *fixed_dofs, long n_fixed, const double *f,
                  double e_min, double pen, double rmin, double volfrac, double move,
                  int precond, double cg_tol, int max_cg, int filter_sens) {
  if (nz > 0 && precond == PC_NODAL) return NULL;
  ocpu *c = (ocpu *)calloc(1, sizeof(ocpu));
  if (!c) return NULL;
  c->nx = nx; c->ny = ny; c->nz = nz > 0 ? nz : 0; c->dim = nz > 0 ? 3 : 2;
  c->dpe = c->dim == 2 ? 8 : 24;
  c->precond = precond; c->max_cg = max_cg;
  c->filter_sens = filter_sens; c->e_min = e_min; c->pen = pen; c->rmin = rmin;
  c->volfrac = volfrac; c->move = move; c->cg_tol = cg_tol; c->alpha_reg = alpha_reg;
  c->nn = (size_t)(nx + 1) * (ny + 1) * (c->dim == 3 ? (size_t)(nz + 1) : 1);
  c->ndof = (size_t)c->dim * c->nn;
  c->ne = (size_t)nx * ny * (c->dim == 3 ? (size_t)nz : 1);
  const size_t km = (size_t)c->dpe * c->dpe;
  c->ke = (double *)malloc(km * sizeof(double));
  c->kinv = (double *)malloc(km * sizeof(double));
  memcpy(c->ke, ke, km * sizeof(double));
  memcpy(c->kinv, kinv, km * sizeof(double));
  const size_t nd = c->ndof, ne = c->ne;
  double **vecs[] = {&c->f, &c->u, &c->r, &c->p, &c->ap, &c->z, &c->diag};
  for (size_t i = 0; i < sizeof(vecs) / sizeof(vecs[0]); ++i)
    *vecs[i] = (double *)calloc(nd, sizeof(double));
  double **evecs[] = {&c->scale, &c->w, &c->rho, &c->rho_phys, &c->dc, &c->dc_filt};
  for (size_t i = 0; i < sizeof(evecs) / sizeof(evecs[0]); ++i)
    *evecs[i] = (double *)calloc(ne, sizeof(double));
  c->tmp = (double *)calloc(nd > ne ? nd : ne, sizeof(double));
  c->binv = (double *)calloc(3 * c->nn, sizeof(double));
  c->fixed = (uint8_t *)calloc(nd, 1);
  for (long i = 0; i < n_fixed; ++i) c->fixed[fixed_dofs[i]] = 1;
  memcpy(c->f, f, nd * sizeof(double));
  for (size_t i = 0; i < nd; ++i)
    if (c->fixed[i]) c->f[i] = 0.0;
  c->f_norm = sqrt(dot(c->f, c->f, nd));
  for (size_t e = 0; e < ne; ++e) c->rho[e] = volfrac;
  return c;
}

void ocpu_destroy(void *h) {
  ocpu *c = (ocpu *)h;
  if (!c) return;
  double *all[] = {c->f, c->u, c->r, c->p, c->ap, c->z, c->diag, c->scale, c->w, c->rho,
                   c->rho_phys, c->dc, c->dc_filt, c->tmp, c->binv};
  for (size_t i = 0; i < sizeof(all) / sizeof(all[0]); ++i) free(all[i]);
  free(c->fixed);
  free(c->ke);
  free(c->kinv);
  free(c);
}

int ocpu_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static double now_s(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

/* One OC iteration (optimizer/simp.py:141-219). out = {compliance, volume,
 * change, cg_iters, cg_status, pcg_seconds, other_seconds}. max_cg_override
 * > 0 bounds this solve (used for bounded timing samples). */
void ocpu_iteration(void *h, int max_cg_override, double out[7]) {
  ocpu *c = (ocpu *)h;
  c->it += 1;
  const int max_cg = c->max_cg;
  if (max_cg_override > 0) c->max_cg = max_cg_override;
  const double t0 = now_s();
  const double *phys = c->rho;
  if (!c->filter_sens) {
    hat_filter(c, c->rho, NULL, c->rho_phys, 0);
    phys = c->rho_phys;
  }
#pragma omp parallel for schedule(static)
  for (long e = 0; e < (long)c->ne; ++e)
    c->scale[e] = c->e_min + pow(phys[e], c->pen) * (1.0 - c->e_min);
  int st = 0;
  const double t1 = now_s();
  const int iters = pcg(c, c->it > 1, &st);
  const double t2 = now_s();
  const double comp = sensitivity(c, phys);
  if (!c->filter_sens) hat_filter(c, c->dc, NULL, c->dc_filt, 0);
  else hat_filter(c, c->dc, c->rho, c->dc_filt, 1);
  double vol = 0.0;
  const double change = oc_update(c, &vol);
  c->max_cg = max_cg;
  const double t3 = now_s();
  out[0] = comp; out[1] = vol; out[2] = change; out[3] = iters; out[4] = st;
  out[5] = t2 - t1; out[6] = (t1 - t0) + (t3 - t2);
}

void ocpu_get_rho(void *h, double *out) {
  ocpu *c = (ocpu *)h;
  memcpy(out, c->rho, c->ne * sizeof(double));
}

void ocpu_set_rho(void *h, const double *in) {
  ocpu *c = (ocpu *)h;
  memcpy(c->rho, in, c->ne * sizeof(double));
}

void ocpu_get_u(void *h, double *out) {
  ocpu *c = (ocpu *)h;
  memcpy(out, c->u, c->ndof * sizeof(double));
}

/* K(rho_phys) p with precomputed SIMP scales from rho (for tests/timing). */
void ocpu_matvec(void *h, const double *rho_phys, const double *p, double *ap) {
  ocpu *c = (ocpu *)h;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < (long)c->ne; ++e)
    c->scale[e] = c->e_min + pow(rho_phys[e], c->pen) * (1.0 - c->e_min);
  matvec(c, p, ap);
}
