// libtpo: host side of the C ABI declared in include/tpo.h.
//
// Single translation unit: the stiffness lives in __constant__ memory, which
// every kernel reads directly.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "design.cuh"
#include "pcg.cuh"
#include "stencil.cuh"
#include "tpo.h"

using namespace tpo;

namespace {

constexpr int kMaxDevices = 64;
constexpr int kStripL = 16;            // node columns per stencil thread
constexpr size_t kAlign = 256;

thread_local std::string g_err;
bool g_have_stiffness[kMaxDevices];
double g_alpha_reg[kMaxDevices];

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define TPO_CK(call)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(TPO_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                    \
  } while (0)

std::atomic<int64_t> g_launches{0};

// after every kernel launch: count it and surface launch errors
#define TPO_CK_LAUNCH()        \
  do {                         \
    g_launches.fetch_add(1);   \
    TPO_CK(cudaGetLastError()); \
  } while (0)

int current_device(int *dev) {
  TPO_CK(cudaGetDevice(dev));
  if (*dev < 0 || *dev >= kMaxDevices) return fail(TPO_ERR_ARGS, "device id %d unsupported", *dev);
  return TPO_OK;
}

int need_stiffness(int *dev) {
  int rc = current_device(dev);
  if (rc) return rc;
  if (!g_have_stiffness[*dev])
    return fail(TPO_ERR_NO_STIFFNESS, "tpo_set_stiffness has not been called on device %d", *dev);
  return TPO_OK;
}

bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// Bump allocator over the caller's workspace (base == nullptr: size query).
struct Carve {
  char *base;
  size_t off = 0;
  explicit Carve(void *b) : base(static_cast<char *>(b)) {}
  template <typename T> T *take(size_t n) {
    off = (off + kAlign - 1) / kAlign * kAlign;
    T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
    off += n * sizeof(T);
    return p;
  }
};

int check_grid(const tpo_grid *g) {
  if (!g) return fail(TPO_ERR_ARGS, "grid is NULL");
  if (g->nelx < 1 || g->nely < 1) return fail(TPO_ERR_ARGS, "nelx, nely must be >= 1");
  if ((int64_t)(g->nelx + 1) * (g->nely + 1) > (int64_t)1 << 30)
    return fail(TPO_ERR_ARGS, "grid too large");
  return TPO_OK;
}

// ----------------------------------------------------------------- launch shapes
struct Shapes {
  dim3 st, up;      // stencil (30-row warps) and pointwise (32-row warps) grids
  int nb_max;       // most CTAs of any PCG kernel
  size_t n_nodes, n_elem;
};

Shapes shapes(const tpo_grid *g) {
  Shapes s;
  const int rows = g->nely + 1, cols = g->nelx + 1;
  const int warps_y = (rows + ROWS_PER_WARP - 1) / ROWS_PER_WARP;
  const int wpb = ST_THREADS / 32;
  s.st = dim3((warps_y + wpb - 1) / wpb, (cols + kStripL - 1) / kStripL, 1);
  s.up = dim3((rows + ST_THREADS - 1) / ST_THREADS, (cols + kStripL - 1) / kStripL, 1);
  s.nb_max = (int)std::max(s.st.x * s.st.y, s.up.x * s.up.y);
  s.n_nodes = (size_t)rows * cols;
  s.n_elem = (size_t)g->nelx * g->nely;
  return s;
}

dim3 flat_grid(size_t n, int threads, int cap) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (size_t)cap) b = cap;
  return dim3((unsigned)b, 1, 1);
}

// ----------------------------------------------------------------- workspace layout
struct PcgWs {
  PcgCtl *ctl;
  OuterCtl *octl;
  double *part;
  double *s64;
  float *s32;
  double *w64;
  float *w32;
  // FP64 solve vectors
  double *ra, *rb, *pa, *pb, *ap, *z;
  // FP32 inner vectors (mixed)
  float *fra, *frb, *fpa, *fpb, *fap, *fz, *fd;
  size_t bytes;
};

PcgWs carve_pcg(void *base, const tpo_grid *g, const tpo_solve_cfg *c) {
  const Shapes sh = shapes(g);
  const size_t N = 2 * sh.n_nodes, E = sh.n_elem;
  const bool block = c->precond == TPO_PRECOND_BLOCK_JACOBI;
  const bool mixed = c->precision == TPO_PRECISION_MIXED;
  Carve cv(base);
  PcgWs w{};
  w.ctl = cv.take<PcgCtl>(1);
  w.octl = cv.take<OuterCtl>(1);
  w.part = cv.take<double>(3 * (size_t)sh.nb_max);
  w.s64 = cv.take<double>(E);
  if (mixed) {
    w.s32 = cv.take<float>(E);
    if (block) w.w32 = cv.take<float>(E);
    w.fra = cv.take<float>(N);
    if (block) w.frb = cv.take<float>(N);
    w.fpa = cv.take<float>(N);
    w.fpb = cv.take<float>(N);
    w.fap = cv.take<float>(N);
    if (block) w.fz = cv.take<float>(N);
    w.fd = cv.take<float>(N);
  } else {
    if (block) w.w64 = cv.take<double>(E);
    w.ra = cv.take<double>(N);
    if (block) w.rb = cv.take<double>(N);
    w.pa = cv.take<double>(N);
    w.pb = cv.take<double>(N);
    w.ap = cv.take<double>(N);
    if (block) w.z = cv.take<double>(N);
  }
  w.bytes = cv.off;
  return w;
}

// ----------------------------------------------------------------- status polling
// Pinned host slots and events used to watch the device status word without
// stalling the launch queue: two chunks of iterations are kept in flight.
struct Poller {
  PcgCtl *host = nullptr;  // 2 pinned slots
  cudaEvent_t ev[2];
  bool ready = false;
};
Poller g_poll[kMaxDevices];
std::mutex g_poll_mu;

int get_poller(Poller **out) {
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_poll_mu);
  Poller &p = g_poll[dev];
  if (!p.ready) {
    TPO_CK(cudaHostAlloc(reinterpret_cast<void **>(&p.host), 2 * sizeof(PcgCtl),
                         cudaHostAllocDefault));
    for (int i = 0; i < 2; ++i)
      TPO_CK(cudaEventCreateWithFlags(&p.ev[i], cudaEventDisableTiming));
    p.ready = true;
  }
  *out = &p;
  return TPO_OK;
}

// ----------------------------------------------------------------- kernel timing
// Opt-in event timing of the PCG kernels (tpo_profile_*). Four events per
// iteration slot (direction start/end, update start/end), created lazily.
constexpr int kProfSlots = 16384;
bool g_prof_on = false;
tpo_profile g_prof{};
std::vector<cudaEvent_t> g_prof_ev[kMaxDevices];

int prof_events(int slots, cudaEvent_t **out) {
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  std::vector<cudaEvent_t> &v = g_prof_ev[dev];
  while ((int)v.size() < 4 * slots) {
    cudaEvent_t e;
    TPO_CK(cudaEventCreate(&e));
    v.push_back(e);
  }
  *out = v.data();
  return TPO_OK;
}

struct LaunchBytes {
  int64_t dir, update;
};

// Runs PCG iterations (direction kernel + update kernel) until the device
// status leaves RUNNING. `iter(slot, ev)` enqueues one iteration; when ev is
// non-null it records ev[0..3] around the two launches.
template <typename IterFn>
int run_iterations(IterFn iter, PcgCtl *dctl, int max_iter, int chunk, cudaStream_t st,
                   PcgCtl *final_out, LaunchBytes lb) {
  Poller *pl;
  int rc = get_poller(&pl);
  if (rc) return rc;
  cudaEvent_t *ev = nullptr;
  const int prof_slots = g_prof_on ? std::min(max_iter, kProfSlots) : 0;
  if (prof_slots > 0 && (rc = prof_events(prof_slots, &ev))) return rc;
  int issued = 0;
  bool pending[2] = {false, false};
  auto issue = [&](int slot) -> int {
    for (int i = 0; i < chunk && issued < max_iter; ++i, ++issued) {
      int r = iter(issued, issued < prof_slots ? ev + 4 * issued : nullptr);
      if (r) return r;
    }
    TPO_CK(cudaMemcpyAsync(&pl->host[slot], dctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaEventRecord(pl->ev[slot], st));
    pending[slot] = true;
    return TPO_OK;
  };
  if (max_iter > 0) {
    if ((rc = issue(0))) return rc;
    if (issued < max_iter && (rc = issue(1))) return rc;
    int cur = 0;
    while (pending[cur]) {
      TPO_CK(cudaEventSynchronize(pl->ev[cur]));
      pending[cur] = false;
      if (pl->host[cur].status != TPO_SOLVE_RUNNING) break;
      if (issued < max_iter && (rc = issue(cur))) return rc;
      cur ^= 1;
    }
  }
  TPO_CK(cudaMemcpyAsync(&pl->host[0], dctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, st));
  TPO_CK(cudaStreamSynchronize(st));
  *final_out = pl->host[0];
  if (prof_slots > 0) {
    // only the launches that did work: the first `it` iterations
    const int real = std::min(final_out->it, std::min(issued, prof_slots));
    for (int i = 0; i < real; ++i) {
      float a = 0.f, b = 0.f;
      TPO_CK(cudaEventElapsedTime(&a, ev[4 * i], ev[4 * i + 1]));
      TPO_CK(cudaEventElapsedTime(&b, ev[4 * i + 2], ev[4 * i + 3]));
      g_prof.dir_ms += a;
      g_prof.update_ms += b;
    }
    g_prof.dir_launches += real;
    g_prof.update_launches += real;
    g_prof.dir_bytes += (int64_t)real * lb.dir;
    g_prof.update_bytes += (int64_t)real * lb.update;
  }
  return TPO_OK;
}

template <typename T, int PRE>
LaunchBytes launch_bytes(const tpo_grid *g) {
  const int64_t nn = (int64_t)(g->nelx + 1) * (g->nely + 1), nd = 2 * nn;
  const int64_t ne = (int64_t)g->nelx * g->nely, s = sizeof(T);
  LaunchBytes lb;
  lb.dir = 4 * nd * s + ne * s + nn;  // r|z, p_old -> p, Ap; scales; mask
  if (PRE == TPO_PRECOND_BLOCK_JACOBI)
    lb.update = 7 * nd * s + ne * s + nn;  // r, Ap, u, p -> u, r', z; weights
  else
    lb.update = 6 * nd * s + (PRE == TPO_PRECOND_NONE ? 0 : ne * s) + nn;  // u, r, p, Ap -> u, r
  return lb;
}

// ----------------------------------------------------------------- FP64 PCG
template <int PRE>
int pcg_fp64(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho, const double *f,
             const uint8_t *fixed, double *u, const PcgWs &w, tpo_solve_result *out,
             cudaStream_t st, double alpha_reg) {
  const Shapes sh = shapes(g);
  const int E = (int)sh.n_elem;
  constexpr bool block = PRE == TPO_PRECOND_BLOCK_JACOBI;
  const double tol_sq = (c->tol * std::sqrt(c->f_norm_sq)) * (c->tol * std::sqrt(c->f_norm_sq));

  k_scales<<<flat_grid(E, 256, 148 * 16), 256, 0, st>>>(E, rho, g->e_min, g->penalty, alpha_reg,
                                                         w.s64, nullptr, block ? w.w64 : nullptr,
                                                         nullptr);
  TPO_CK_LAUNCH();
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, 0.0, c->max_iter, nullptr, 0.0);
  TPO_CK_LAUNCH();
  if (!c->warm_start) TPO_CK(cudaMemsetAsync(u, 0, 2 * sh.n_nodes * sizeof(double), st));

  StArgs a{};
  a.nx = g->nelx;
  a.ny = g->nely;
  a.s = w.s64;
  a.fixed = fixed;
  a.in = u;
  a.uw = u;
  a.f = f;
  a.out = w.ra;
  a.part = w.part;
  a.ctl = w.ctl;
  k_stencil<double, M_RES, PRE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(a);
  TPO_CK_LAUNCH();

  BlkArgs b{};
  b.nx = g->nelx;
  b.ny = g->nely;
  b.w = w.w64;
  b.fixed = fixed;
  b.u = u;
  b.ap = w.ap;
  b.pa = w.pa;
  b.pb = w.pb;
  b.ra = w.ra;
  b.rb = w.rb;
  b.z = w.z;
  b.part = w.part;
  b.ctl = w.ctl;
  if (block) {
    k_blockpre<double, true, kStripL><<<sh.st, ST_THREADS, 0, st>>>(b);
    TPO_CK_LAUNCH();
  }

  StArgs d{};
  d.nx = g->nelx;
  d.ny = g->nely;
  d.s = w.s64;
  d.fixed = fixed;
  d.out = w.ap;
  d.r = w.ra;
  d.z = w.z;
  d.pa = w.pa;
  d.pb = w.pb;
  d.part = w.part;
  d.ctl = w.ctl;
  UpdArgs up{};
  up.nx = g->nelx;
  up.ny = g->nely;
  up.s = w.s64;
  up.fixed = fixed;
  up.u = u;
  up.r = w.ra;
  up.ap = w.ap;
  up.pa = w.pa;
  up.pb = w.pb;
  up.part = w.part;
  up.ctl = w.ctl;

  auto iter = [&](int, cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    k_stencil<double, M_DIR, PRE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(d);
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    if (ev) TPO_CK(cudaEventRecord(ev[2], st));
    if (block) {
      k_blockpre<double, false, kStripL><<<sh.st, ST_THREADS, 0, st>>>(b);
    } else {
      k_update<double, PRE, kStripL><<<sh.up, ST_THREADS, 0, st>>>(up);
    }
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[3], st));
    return TPO_OK;
  };
  PcgCtl fin;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  int rc = run_iterations(iter, w.ctl, c->max_iter, chunk, st, &fin,
                          launch_bytes<double, PRE>(g));
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

// ----------------------------------------------------------------- mixed PCG
template <int PRE>
int pcg_mixed(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho, const double *f,
              const uint8_t *fixed, double *u, const PcgWs &w, tpo_solve_result *out,
              cudaStream_t st, double alpha_reg) {
  const Shapes sh = shapes(g);
  const int E = (int)sh.n_elem;
  constexpr bool block = PRE == TPO_PRECOND_BLOCK_JACOBI;
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);

  k_scales<<<flat_grid(E, 256, 148 * 16), 256, 0, st>>>(E, rho, g->e_min, g->penalty, alpha_reg,
                                                         w.s64, w.s32, nullptr,
                                                         block ? w.w32 : nullptr);
  TPO_CK_LAUNCH();
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, 0.0, c->inner_tol * c->inner_tol, c->max_iter, w.octl,
                              tol_sq);
  TPO_CK_LAUNCH();
  if (!c->warm_start) TPO_CK(cudaMemsetAsync(u, 0, 2 * sh.n_nodes * sizeof(double), st));

  StArgs rx{};
  rx.nx = g->nelx;
  rx.ny = g->nely;
  rx.s = w.s64;
  rx.fixed = fixed;
  rx.in = u;
  rx.uw = u;
  rx.f = f;
  rx.out = w.fra;
  rx.d = w.fd;
  rx.part = w.part;
  rx.ctl = w.ctl;
  rx.octl = w.octl;

  BlkArgs b{};
  b.nx = g->nelx;
  b.ny = g->nely;
  b.w = w.w32;
  b.fixed = fixed;
  b.u = w.fd;
  b.ap = w.fap;
  b.pa = w.fpa;
  b.pb = w.fpb;
  b.ra = w.fra;
  b.rb = w.frb;
  b.z = w.fz;
  b.part = w.part;
  b.ctl = w.ctl;

  StArgs d{};
  d.nx = g->nelx;
  d.ny = g->nely;
  d.s = w.s32;
  d.fixed = fixed;
  d.out = w.fap;
  d.r = w.fra;
  d.z = w.fz;
  d.pa = w.fpa;
  d.pb = w.fpb;
  d.part = w.part;
  d.ctl = w.ctl;
  UpdArgs up{};
  up.nx = g->nelx;
  up.ny = g->nely;
  up.s = w.s32;
  up.fixed = fixed;
  up.u = w.fd;
  up.r = w.fra;
  up.ap = w.fap;
  up.pa = w.fpa;
  up.pb = w.fpb;
  up.part = w.part;
  up.ctl = w.ctl;

  auto iter = [&](int, cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    k_stencil<float, M_DIR, PRE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(d);
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    if (ev) TPO_CK(cudaEventRecord(ev[2], st));
    if (block) {
      k_blockpre<float, false, kStripL><<<sh.st, ST_THREADS, 0, st>>>(b);
    } else {
      k_update<float, PRE, kStripL><<<sh.up, ST_THREADS, 0, st>>>(up);
    }
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[3], st));
    return TPO_OK;
  };

  Poller *pl;
  int rc = get_poller(&pl);
  if (rc) return rc;
  OuterCtl oh{};
  int total_inner = 0, outer_steps = 0, status = TPO_SOLVE_MAX_ITER;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  for (int k = 0;; ++k) {
    k_stencil<double, M_RESX, PRE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(rx);
    TPO_CK_LAUNCH();
    if (block) {
      k_blockpre<float, true, kStripL><<<sh.st, ST_THREADS, 0, st>>>(b);
      TPO_CK_LAUNCH();
    }
    TPO_CK(cudaMemcpyAsync(&oh, w.octl, sizeof(OuterCtl), cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaStreamSynchronize(st));
    if (oh.status != TPO_SOLVE_RUNNING) {
      status = oh.status;
      break;
    }
    if (k >= c->max_outer) {
      status = TPO_SOLVE_MAX_ITER;
      break;
    }
    PcgCtl fin;
    rc = run_iterations(iter, w.ctl, c->max_iter, chunk, st, &fin, launch_bytes<float, PRE>(g));
    if (rc) return rc;
    total_inner += fin.it;
    ++outer_steps;
    if (fin.status == TPO_SOLVE_NONFINITE) {
      status = TPO_SOLVE_NONFINITE;
      break;
    }
    k_correct<<<flat_grid(2 * sh.n_nodes, 256, 148 * 16), 256, 0, st>>>(2 * sh.n_nodes, u, w.fd);
    TPO_CK_LAUNCH();
  }
  TPO_CK(cudaStreamSynchronize(st));
  out->status = status;
  out->iters = total_inner;
  out->updates = total_inner;
  out->outer_iters = outer_steps;
  out->rr = oh.rr;
  return TPO_OK;
}


}  // namespace

template <typename T>
static int matvec_impl(const tpo_grid *g, const T *rho, const uint8_t *fixed, const T *p, T *ap,
                       double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!rho || !fixed || !p || !ap || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(p, 2 * sizeof(T)) || !aligned(ap, 2 * sizeof(T)) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer");
  if (ws_bytes < tpo_matvec_workspace_bytes(g))
    return fail(TPO_ERR_WORKSPACE, "workspace too small");
  const Shapes sh = shapes(g);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  Carve cv(ws);
  PcgCtl *ctl = cv.take<PcgCtl>(1);
  double *part = cv.take<double>((size_t)sh.nb_max);
  T *sc = cv.take<T>(sh.n_elem);
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(PcgCtl), st));
  k_scales_t<T><<<flat_grid(sh.n_elem, 256, 148 * 16), 256, 0, st>>>((int)sh.n_elem, rho,
                                                                       g->e_min, g->penalty, sc);
  TPO_CK_LAUNCH();
  StArgs a{};
  a.nx = g->nelx;
  a.ny = g->nely;
  a.s = sc;
  a.fixed = fixed;
  a.in = p;
  a.out = ap;
  a.part = part;
  a.ctl = ctl;
  a.result = pap_out;
  k_stencil<T, M_RAW, TPO_PRECOND_NONE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(a);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

template <typename T>
static int apply_impl(const tpo_grid *g, const T *scale, const uint8_t *fixed, const T *p, T *ap,
                      double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!scale || !fixed || !p || !ap || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(p, 2 * sizeof(T)) || !aligned(ap, 2 * sizeof(T)) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer");
  if (ws_bytes < tpo_matvec_workspace_bytes(g))
    return fail(TPO_ERR_WORKSPACE, "workspace too small");
  const Shapes sh = shapes(g);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  Carve cv(ws);
  PcgCtl *ctl = cv.take<PcgCtl>(1);
  double *part = cv.take<double>((size_t)sh.nb_max);
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(PcgCtl), st));
  StArgs a{};
  a.nx = g->nelx;
  a.ny = g->nely;
  a.s = scale;
  a.fixed = fixed;
  a.in = p;
  a.out = ap;
  a.part = part;
  a.ctl = ctl;
  a.result = pap_out;
  k_stencil<T, M_RAW, TPO_PRECOND_NONE, kStripL><<<sh.st, ST_THREADS, 0, st>>>(a);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// =================================================================== C ABI
extern "C" {

int tpo_version(void) { return 1; }

const char *tpo_last_error_string(void) { return g_err.c_str(); }

int tpo_set_stiffness(const double ke[64], const double ke_inv[64], double alpha_reg) {
  if (!ke || !ke_inv) return fail(TPO_ERR_ARGS, "ke and ke_inv must be non-NULL");
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  float kf[64], kif[64];
  for (int i = 0; i < 64; ++i) {
    kf[i] = (float)ke[i];
    kif[i] = (float)ke_inv[i];
  }
  TPO_CK(cudaMemcpyToSymbol(c_ke, ke, sizeof(double) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_ke_f, kf, sizeof(float) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_kinv, ke_inv, sizeof(double) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_kinv_f, kif, sizeof(float) * 64));
  g_alpha_reg[dev] = alpha_reg;
  g_have_stiffness[dev] = true;
  return TPO_OK;
}

// ------------------------------------------------------------------ matvec
size_t tpo_matvec_workspace_bytes(const tpo_grid *g) {
  if (check_grid(g)) return 0;
  const Shapes sh = shapes(g);
  Carve cv(nullptr);
  cv.take<PcgCtl>(1);
  cv.take<double>((size_t)sh.nb_max);
  cv.take<double>(sh.n_elem);
  return cv.off;
}

int tpo_matvec_f64(const tpo_grid *g, const double *rho, const uint8_t *fixed, const double *p,
                   double *ap, double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  return matvec_impl<double>(g, rho, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_matvec_f32(const tpo_grid *g, const float *rho, const uint8_t *fixed, const float *p,
                   float *ap, double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  return matvec_impl<float>(g, rho, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_apply_stiffness_f64(const tpo_grid *g, const double *scale, const uint8_t *fixed,
                            const double *p, double *ap, double *pap_out, void *ws,
                            size_t ws_bytes, tpo_stream s) {
  return apply_impl<double>(g, scale, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_apply_stiffness_f32(const tpo_grid *g, const float *scale, const uint8_t *fixed,
                            const float *p, float *ap, double *pap_out, void *ws,
                            size_t ws_bytes, tpo_stream s) {
  return apply_impl<float>(g, scale, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

// ------------------------------------------------------------------ profiling
int tpo_profile_enable(int on) {
  g_prof_on = on != 0;
  return TPO_OK;
}

int tpo_profile_reset(void) {
  g_prof = tpo_profile{};
  g_launches.store(0);
  return TPO_OK;
}

int tpo_profile_read(tpo_profile *out) {
  if (!out) return fail(TPO_ERR_ARGS, "NULL profile");
  *out = g_prof;
  out->launches = g_launches.load();
  return TPO_OK;
}

// ------------------------------------------------------------------ PCG
size_t tpo_pcg_workspace_bytes(const tpo_grid *g, const tpo_solve_cfg *c) {
  if (check_grid(g) || !c) return 0;
  return carve_pcg(nullptr, g, c).bytes;
}

int tpo_pcg_solve(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho_phys,
                  const double *f, const uint8_t *fixed, double *u, void *ws, size_t ws_bytes,
                  tpo_solve_result *out, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!c || !out) return fail(TPO_ERR_ARGS, "cfg and result must be non-NULL");
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!rho_phys || !f || !fixed || !u || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(f, 16) || !aligned(u, 16) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer (nodal vectors need 16 B, workspace 256 B)");
  if (c->precond < TPO_PRECOND_NONE || c->precond > TPO_PRECOND_NODAL_BLOCK)
    return fail(TPO_ERR_ARGS, "unknown preconditioner %d", c->precond);
  if (c->precision != TPO_PRECISION_FP64 && c->precision != TPO_PRECISION_MIXED)
    return fail(TPO_ERR_ARGS, "unknown precision %d", c->precision);
  if (!(c->tol >= 0.0) || !(c->f_norm_sq >= 0.0))
    return fail(TPO_ERR_ARGS, "tol and f_norm_sq must be >= 0");
  const PcgWs w = carve_pcg(ws, g, c);
  if (ws_bytes < w.bytes) return fail(TPO_ERR_WORKSPACE, "workspace %zu < %zu", ws_bytes, w.bytes);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  memset(out, 0, sizeof(*out));

  // reference solver.py:59-63: ||f|| < 1e-30 -> u = 0, no iterations
  if (std::sqrt(c->f_norm_sq) < 1e-30) {
    const Shapes sh = shapes(g);
    TPO_CK(cudaMemsetAsync(u, 0, 2 * sh.n_nodes * sizeof(double), st));
    TPO_CK(cudaStreamSynchronize(st));
    out->status = TPO_SOLVE_ZERO_RHS;
    return TPO_OK;
  }
  const double ar = g_alpha_reg[dev];
  const bool mixed = c->precision == TPO_PRECISION_MIXED;
  switch (c->precond) {
    case TPO_PRECOND_NONE:
      return mixed ? pcg_mixed<TPO_PRECOND_NONE>(g, c, rho_phys, f, fixed, u, w, out, st, ar)
                   : pcg_fp64<TPO_PRECOND_NONE>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    case TPO_PRECOND_JACOBI:
      return mixed ? pcg_mixed<TPO_PRECOND_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar)
                   : pcg_fp64<TPO_PRECOND_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    case TPO_PRECOND_BLOCK_JACOBI:
      return mixed
                 ? pcg_mixed<TPO_PRECOND_BLOCK_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar)
                 : pcg_fp64<TPO_PRECOND_BLOCK_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    default:
      return mixed
                 ? pcg_mixed<TPO_PRECOND_NODAL_BLOCK>(g, c, rho_phys, f, fixed, u, w, out, st, ar)
                 : pcg_fp64<TPO_PRECOND_NODAL_BLOCK>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
  }
}

// ------------------------------------------------------------------ sensitivity
size_t tpo_sensitivity_workspace_bytes(const tpo_grid *g) {
  if (check_grid(g)) return 0;
  const dim3 gr((g->nely + S_THREADS - 1) / S_THREADS, (g->nelx + SL - 1) / SL, 1);
  Carve cv(nullptr);
  cv.take<SumCtl>(1);
  cv.take<double>((size_t)gr.x * gr.y);
  return cv.off;
}

int tpo_sensitivity(const tpo_grid *g, const double *rho_phys, const double *u, double *dc,
                    double *compliance_out, void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!rho_phys || !u || !dc || !compliance_out || !ws)
    return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(u, 16) || !aligned(ws, kAlign)) return fail(TPO_ERR_ARGS, "misaligned pointer");
  if (ws_bytes < tpo_sensitivity_workspace_bytes(g))
    return fail(TPO_ERR_WORKSPACE, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  const dim3 gr((g->nely + S_THREADS - 1) / S_THREADS, (g->nelx + SL - 1) / SL, 1);
  Carve cv(ws);
  SumCtl *ctl = cv.take<SumCtl>(1);
  double *part = cv.take<double>((size_t)gr.x * gr.y);
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(SumCtl), st));
  k_sensitivity<<<gr, S_THREADS, 0, st>>>(g->nelx, g->nely, g->e_min, g->penalty, rho_phys, u, dc,
                                          part, ctl, compliance_out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// ------------------------------------------------------------------ sensitivity, no allocation
// Scratch for tpo_sensitivity_noalloc: the completion ticket (first 256 bytes)
// and the per-CTA partial sums. Host code must not take this name as a device
// address; the address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_sens_scratch[TPO_SENS_NOALLOC_SCRATCH];
static constexpr size_t kSensTicketBytes = 256;
static constexpr size_t kSensMaxPartials =
    (TPO_SENS_NOALLOC_SCRATCH - kSensTicketBytes) / sizeof(double);
static void *g_sens_scratch_addr[kMaxDevices];
static std::mutex g_sens_scratch_mu;

int tpo_sensitivity_noalloc(const tpo_grid *g, const double *rho_phys, const double *u,
                            double *dc, double *compliance_out, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!rho_phys || !u || !dc || !compliance_out) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(u, 16)) return fail(TPO_ERR_ARGS, "misaligned pointer");
  const dim3 gr((g->nely + S_THREADS - 1) / S_THREADS, (g->nelx + SL - 1) / SL, 1);
  const size_t nb = (size_t)gr.x * gr.y;
  if (nb > kSensMaxPartials)
    return fail(TPO_ERR_ARGS,
                "grid %dx%d needs %zu partial sums; the fixed scratch holds %zu "
                "(ceil(nely/128)*ceil(nelx/16) must be <= %zu)",
                g->nelx, g->nely, nb, kSensMaxPartials, kSensMaxPartials);
  void *base;
  {
    std::lock_guard<std::mutex> lk(g_sens_scratch_mu);
    if (!g_sens_scratch_addr[dev]) {
      void *ptr = nullptr;
      TPO_CK(cudaGetSymbolAddress(&ptr, g_sens_scratch));
      g_sens_scratch_addr[dev] = ptr;
    }
    base = g_sens_scratch_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(s);
  SumCtl *ctl = static_cast<SumCtl *>(base);
  double *part = reinterpret_cast<double *>(static_cast<unsigned char *>(base) + kSensTicketBytes);
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(SumCtl), st));  // the ticket must start at zero
  k_sensitivity<<<gr, S_THREADS, 0, st>>>(g->nelx, g->nely, g->e_min, g->penalty, rho_phys, u, dc,
                                          part, ctl, compliance_out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// ------------------------------------------------------------------ filters
static int filter_launch(const tpo_grid *g, double rmin, int mode, const double *x,
                         const double *rho, double *out, double *s_out, float *s32_out,
                         tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!x || !out || (mode == F_SENS && !rho)) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!(rmin > 0.0)) return fail(TPO_ERR_ARGS, "rmin must be > 0");
  const int R = (int)std::ceil(rmin);
  if (R > F_MAXR) return fail(TPO_ERR_ARGS, "ceil(rmin) = %d exceeds %d", R, F_MAXR);
  const int W = 2 * R + 1, TW = FT + 2 * R;
  const size_t smem = (size_t)(W * W + TW * TW) * sizeof(double);
  const dim3 gr((g->nely + FT - 1) / FT, (g->nelx + FT - 1) / FT, 1);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  if (mode == F_DENSITY) {
    k_filter<F_DENSITY><<<gr, F_THREADS, smem, st>>>(g->nelx, g->nely, rmin, R, x, rho, out, s_out,
                                                     s32_out, g->e_min, g->penalty);
  } else {
    k_filter<F_SENS><<<gr, F_THREADS, smem, st>>>(g->nelx, g->nely, rmin, R, x, rho, out, nullptr,
                                                  nullptr, g->e_min, g->penalty);
  }
  TPO_CK_LAUNCH();
  return TPO_OK;
}

int tpo_density_filter(const tpo_grid *g, double rmin, const double *x, double *out,
                       double *scale_out, float *scale32_out, tpo_stream s) {
  return filter_launch(g, rmin, F_DENSITY, x, nullptr, out, scale_out, scale32_out, s);
}

int tpo_sensitivity_filter(const tpo_grid *g, double rmin, const double *rho, const double *dc,
                           double *out, tpo_stream s) {
  return filter_launch(g, rmin, F_SENS, dc, rho, out, nullptr, nullptr, s);
}

// ------------------------------------------------------------------ OC
static dim3 oc_grid(size_t n) { return flat_grid(n, OC_THREADS, 148 * 4); }

size_t tpo_oc_workspace_bytes(const tpo_grid *g) {
  if (check_grid(g)) return 0;
  const dim3 gr = oc_grid((size_t)g->nelx * g->nely);
  Carve cv(nullptr);
  cv.take<OcCtl>(1);
  cv.take<double>(2 * (size_t)gr.x);
  return cv.off;
}

int tpo_oc_update(const tpo_grid *g, double volfrac, double move, const double *rho_in,
                  const double *dc, const double *dv, double *rho_out, double *result_out,
                  void *ws, size_t ws_bytes, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!rho_in || !dc || !rho_out || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(ws, kAlign)) return fail(TPO_ERR_ARGS, "misaligned workspace");
  if (ws_bytes < tpo_oc_workspace_bytes(g)) return fail(TPO_ERR_WORKSPACE, "workspace too small");
  const size_t n = (size_t)g->nelx * g->nely;
  const dim3 gr = oc_grid(n);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  Carve cv(ws);
  OcCtl *ctl = cv.take<OcCtl>(1);
  double *part = cv.take<double>(2 * (size_t)gr.x);
  k_oc_init<<<1, 1, 0, st>>>(ctl);
  TPO_CK_LAUNCH();
  for (int i = 0; i < OC_MAX_STEPS; ++i) {
    k_oc_step<<<gr, OC_THREADS, 0, st>>>((int)n, volfrac, move, rho_in, dc, dv, part, ctl);
    TPO_CK_LAUNCH();
  }
  k_oc_final<<<gr, OC_THREADS, 0, st>>>((int)n, move, rho_in, dc, dv, rho_out, ctl, result_out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

}  // extern "C"
