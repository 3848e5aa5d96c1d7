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
#include "cgstep.cuh"
#include "hex3d.cuh"
#include "stencil.cuh"
#include "tpo.h"

using namespace tpo;

namespace {

constexpr int kMaxDevices = 64;
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

// The bilinear plane-stress Ke of a unit square splits exactly into a centre
// (one-point) part and a rank-2 hourglass part:
//   Ke = B0^T D B0 + ch (hx hx^T + hy hy^T),
//   B0 = strain-displacement matrix at the element centre
//        (dN/dx = (-1, 1, 1, -1)/2, dN/dy = (-1, -1, 1, 1)/2 per corner),
//   D  = [[d11, d12, 0], [d12, d11, 0], [0, 0, d33]],  hx, hy = (1, -1, 1, -1)
//   on the x (y) DOFs of the corners.
// The stencil applies Ke in that form (about 40 flops per element instead of
// 64 multiply-adds). The four constants are read off Ke's entries and the
// decomposition is checked against every entry; a Ke that does not have this
// structure is rejected. kst = {d11/4, d12/4, d33/4, ch}.
int stiffness_structure(const double ke[64], double kst[6]) {
  const double ch = 0.5 * (ke[0] + ke[4]);
  const double d12 = 2.0 * (ke[1] + ke[3]);
  const double d33 = 2.0 * (ke[1] - ke[3]);
  const double d11 = 2.0 * (ke[0] - ke[4]) - d33;
  const double dnx[4] = {-0.5, 0.5, 0.5, -0.5}, dny[4] = {-0.5, -0.5, 0.5, 0.5};
  const double h[4] = {1.0, -1.0, 1.0, -1.0};
  double b[3][8] = {};
  for (int i = 0; i < 4; ++i) {
    b[0][2 * i] = dnx[i];
    b[1][2 * i + 1] = dny[i];
    b[2][2 * i] = dny[i];
    b[2][2 * i + 1] = dnx[i];
  }
  const double d[3][3] = {{d11, d12, 0.0}, {d12, d11, 0.0}, {0.0, 0.0, d33}};
  double scale = 0.0, err = 0.0;
  for (int i = 0; i < 64; ++i) scale = fmax(scale, fabs(ke[i]));
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      double v = 0.0;
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) v += b[p][i] * d[p][q] * b[q][j];
      if ((i & 1) == (j & 1)) v += ch * h[i / 2] * h[j / 2];
      err = fmax(err, fabs(v - ke[8 * i + j]));
    }
  if (!(scale > 0.0) || !(err <= 1e-12 * scale))
    return fail(TPO_ERR_ARGS,
                "ke is not the bilinear plane-stress element of a unit square "
                "(structure mismatch %.3e of max entry %.3e)", err, scale);
  kst[0] = 0.25 * d11;
  kst[1] = 0.25 * d12;
  kst[2] = 0.25 * d33;
  kst[3] = ch;
  kst[4] = ke[0];  // every diagonal entry (checked above through the structure)
  kst[5] = ke[1];  // x-y entry of corner 0; corners 1..3 alternate in sign
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

// ----------------------------------------------------------------- launch plans
dim3 flat_grid(size_t n, int threads, int cap) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > (size_t)cap) b = cap;
  return dim3((unsigned)b, 1, 1);
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
  }
  return n;
}

// Stencil launch configuration per kernel instantiation: dynamic shared
// memory (set once), resident CTAs per SM, and the strip length that makes
// the grid close to one full wave.
// failure tests (tpo_test_withhold_stage): group + 1 for the next stencil launch
std::atomic<int> g_withhold1{0};

#ifndef TPO_MIN_STRIP
#define TPO_MIN_STRIP 8
#endif
#ifndef TPO_ST_G
#define TPO_ST_G 2  // stencil columns per ring slot
#endif
#ifndef TPO_ST_NG
#define TPO_ST_NG 4  // ring slots
#endif
constexpr int kMinStrip = TPO_MIN_STRIP;  // shortest stencil strip (node columns)
template <typename T, typename C, int MODE, int PRE> struct StencilCfg {
  static constexpr int G = TPO_ST_G;
  static constexpr int NG = TPO_ST_NG;
  static constexpr int SMEM = TsGeom<T, MODE>::template slot_bytes<G>() * NG;
  static int resident() {
    static int occ = -1;
    if (occ < 0) {
      auto kern = k_tstencil<T, C, MODE, PRE, G, NG>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
      int o = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, TS_THREADS, SMEM) !=
              cudaSuccess || o < 1)
        o = 1;
      occ = o;
    }
    return occ;
  }
  struct Plan {
    dim3 grid;
    int L;
  };
  static Plan plan(int nx, int ny) {
    const int rows = (ny + 1 + RPC - 1) / RPC;
    const int target = sm_count() * resident();
    int strips = std::max(1, target / rows);
    int L = std::max(kMinStrip, (nx + 1 + strips - 1) / strips);
    strips = (nx + 1 + L - 1) / L;
    return Plan{dim3(rows, strips, 1), L};
  }
  static int launch(cudaStream_t st, const TsArgs &a, int nx, int ny) {
    const Plan pl = plan(nx, ny);
    TsArgs b = a;
    b.withhold1 = g_withhold1.exchange(0);  // 0 unless a failure test armed it
    k_tstencil<T, C, MODE, PRE, G, NG><<<pl.grid, TS_THREADS, SMEM, st>>>(b, pl.L);
    return TPO_OK;
  }
  static int max_ctas(int nx, int ny) {
    const Plan pl = plan(nx, ny);
    return (int)(pl.grid.x * pl.grid.y);
  }
};

// Launch configuration of the one-launch iteration (k_cgstep): a ring of NG
// staged columns per CTA (3 x 11 KB in FP64: six CTAs fit an SM), a grid of
// about one full wave.
template <typename T, typename C, int PRE> struct CgCfg {
  static constexpr int NG = 3;
  static constexpr int SMEM = CgGeom<T>::SLOT * NG;
  static int resident() {
    static int occ = -1;
    if (occ < 0) {
      auto kern = k_cgstep<T, C, PRE, NG>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
      int o = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, CG_THREADS, SMEM) !=
              cudaSuccess || o < 1)
        o = 1;
      occ = o;
    }
    return occ;
  }
  static void plan(int nx, int ny, dim3 *grid, int *L) {
    const int rows = (ny + 1 + RPC - 1) / RPC;
    const int target = sm_count() * resident();
    int strips = std::max(1, target / rows);
    int l = std::max(8, (nx + 1 + strips - 1) / strips);
    strips = (nx + 1 + l - 1) / l;
    *grid = dim3(rows, strips, 1);
    *L = l;
  }
  static void launch(cudaStream_t st, const CgArgs &a, int nx, int ny) {
    dim3 grid;
    int L;
    plan(nx, ny, &grid, &L);
    k_cgstep<T, C, PRE, NG><<<grid, CG_THREADS, SMEM, st>>>(a, L);
  }
};

// flat update: runs of UQ rows, one per thread, at most eight 256-thread CTAs
// per SM (this bound sizes the partial-sum buffers); grid-stride beyond
int update_flat_ctas(int nx, int ny) {
  const int64_t total = (int64_t)(nx + 1) * ((ny + 1 + UQ - 1) / UQ);
  const int64_t want = (total + UF_THREADS - 1) / UF_THREADS;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count() * 8));
}
// the launched grid: one wave of the kernel's resident CTAs, within that bound
template <auto KERN> int flat_wave(int nx, int ny) {
  static int occ = -1;
  if (occ < 0) {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, KERN, UF_THREADS, 0) != cudaSuccess ||
        o < 1)
      o = 1;
    occ = o;
  }
  return std::min(update_flat_ctas(nx, ny), sm_count() * occ);
}
constexpr int kBlkL = 16;
dim3 blk_grid(int nx, int ny) {
  const int warps_y = (ny + 1 + RPW - 1) / RPW;
  return dim3((warps_y + WPC - 1) / WPC, (nx + 1 + kBlkL - 1) / kBlkL, 1);
}

// most CTAs any PCG kernel of this grid can have (sizes the partials buffer)
int max_ctas(const tpo_grid *g) {
  const int nx = g->nelx, ny = g->nely;
  int m = update_flat_ctas(nx, ny);
  const dim3 bg = blk_grid(nx, ny);
  m = std::max(m, (int)(bg.x * bg.y));
  // the stencil plans target at most sm_count * 8 CTAs (resident <= 8 with 128 threads
  // and >= 37 KB of shared memory); bound generously without querying every variant
  const int rows = (ny + 1 + RPC - 1) / RPC;
  m = std::max(m, rows * std::max(1, (nx + 1 + 7) / 8));
  return m;
}

// ----------------------------------------------------------------- workspace layout
struct PcgWs {
  PcgCtl *ctl;
  OuterCtl *octl;
  double *part;
  uint8_t *mask;
  double *u, *f;          // padded FP64 solution and load
  double *s64, *w64;
  float *s32, *w32;
  double *ra, *rb, *pa, *pb, *ap, *z;          // FP64 solve
  float *fra, *frb, *fpa, *fpb, *fap, *fz;       // mixed: FP32 Krylov vectors (u stays FP64)
  double *wa, *wb, *sa, *sb;                   // one-launch form: w = K M^-1 r, s = K p
  bool single;                                 // one launch per iteration (k_cgstep)
  uint32_t *bodies;                            // asynchronous solve: loop bodies run
  int P;
  size_t bytes;
};

// The one-launch iteration serves the plain FP64 solve with a point
// preconditioner (its s = K p recurrence is not kept accurately in FP32).
bool use_single(const tpo_solve_cfg *c) {
  return c->precond != TPO_PRECOND_BLOCK_JACOBI && c->precision == TPO_PRECISION_FP64 &&
         c->recurrence != TPO_RECURRENCE_STANDARD;
}

PcgWs carve_pcg(void *base, const tpo_grid *g, const tpo_solve_cfg *c) {
  const int nx = g->nelx, ny = g->nely, P = pad_pitch(ny);
  const size_t NN = (size_t)(nx + 1) * P, NE = (size_t)nx * P;
  const bool block = c->precond == TPO_PRECOND_BLOCK_JACOBI;
  const bool mixed = c->precision == TPO_PRECISION_MIXED;
  Carve cv(base);
  PcgWs w{};
  w.P = P;
  w.ctl = cv.take<PcgCtl>(1);
  w.octl = cv.take<OuterCtl>(1);
  w.bodies = cv.take<uint32_t>(1);
  w.part = cv.take<double>(3 * (size_t)max_ctas(g));  // up to 3 sums per CTA
  w.mask = cv.take<uint8_t>(NN);
  w.u = cv.take<double>(2 * NN);
  w.f = cv.take<double>(2 * NN);
  w.s64 = cv.take<double>(NE);
  w.single = use_single(c);
  if (w.single) {
    // r, w, s ping-pong; p in place; the solution is u itself
    w.ra = cv.take<double>(2 * NN);
    w.rb = cv.take<double>(2 * NN);
    w.wa = cv.take<double>(2 * NN);
    w.wb = cv.take<double>(2 * NN);
    w.sa = cv.take<double>(2 * NN);
    w.sb = cv.take<double>(2 * NN);
    w.pa = cv.take<double>(2 * NN);
  } else if (mixed) {
    w.s32 = cv.take<float>(NE);
    if (block) w.w32 = cv.take<float>(NE);
    w.fra = cv.take<float>(2 * NN);
    if (block) w.frb = cv.take<float>(2 * NN);
    w.fpa = cv.take<float>(2 * NN);
    w.fpb = cv.take<float>(2 * NN);
    w.fap = cv.take<float>(2 * NN);
    w.fz = cv.take<float>(2 * NN);  // z (the element-block z, or M r stored by the update)
  } else {
    if (block) w.w64 = cv.take<double>(NE);
    w.ra = cv.take<double>(2 * NN);
    if (block) w.rb = cv.take<double>(2 * NN);
    w.pa = cv.take<double>(2 * NN);
    w.pb = cv.take<double>(2 * NN);
    w.ap = cv.take<double>(2 * NN);
    w.z = cv.take<double>(2 * NN);
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
  int64_t step = 0;  // nonzero: one launch per iteration, timed by ev[0..1]
};

// Runs PCG iterations (direction kernel + update kernel) until the device
// status leaves RUNNING. `iter(ev)` enqueues one iteration; when ev is
// non-null it records ev[0..3] around the two launches. it0 = the device
// iteration count when this call starts.
template <typename IterFn>
int run_iterations(IterFn iter, PcgCtl *dctl, int max_iter, int it0, int chunk, cudaStream_t st,
                   PcgCtl *final_out, LaunchBytes lb) {
  Poller *pl;
  int rc = get_poller(&pl);
  if (rc) return rc;
  cudaEvent_t *ev = nullptr;
  const int budget = std::max(0, max_iter - it0);
  const int prof_slots = g_prof_on ? std::min(budget, kProfSlots) : 0;
  if (prof_slots > 0 && (rc = prof_events(prof_slots, &ev))) return rc;
  int issued = 0;
  bool pending[2] = {false, false};
  auto issue = [&](int slot) -> int {
    for (int i = 0; i < chunk && issued < budget; ++i, ++issued) {
      int r = iter(issued < prof_slots ? ev + 4 * issued : nullptr);
      if (r) return r;
    }
    TPO_CK(cudaMemcpyAsync(&pl->host[slot], dctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaEventRecord(pl->ev[slot], st));
    pending[slot] = true;
    return TPO_OK;
  };
  if (budget > 0) {
    if ((rc = issue(0))) return rc;
    if (issued < budget && (rc = issue(1))) return rc;
    int cur = 0;
    while (pending[cur]) {
      TPO_CK(cudaEventSynchronize(pl->ev[cur]));
      pending[cur] = false;
      if (pl->host[cur].status != TPO_SOLVE_RUNNING || pl->host[cur].err) break;
      if (issued < budget && (rc = issue(cur))) return rc;
      cur ^= 1;
    }
  }
  TPO_CK(cudaMemcpyAsync(&pl->host[0], dctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, st));
  TPO_CK(cudaStreamSynchronize(st));
  *final_out = pl->host[0];
  if (final_out->err) return fail(TPO_ERR_TIMEOUT, "a TMA pipeline wait ran out of time");
  if (prof_slots > 0) {
    // only the launches that did work
    const int real = std::min(final_out->it - it0, std::min(issued, prof_slots));
    if (lb.step > 0) {
      for (int i = 0; i < real; ++i) {
        float a = 0.f;
        TPO_CK(cudaEventElapsedTime(&a, ev[4 * i], ev[4 * i + 1]));
        g_prof.step_ms += a;
      }
      if (real > 0) {
        g_prof.step_launches += real;
        g_prof.step_bytes += (int64_t)real * lb.step;
      }
    }
    for (int i = 0; i < real && lb.step == 0; ++i) {
      float a = 0.f, b = 0.f;
      TPO_CK(cudaEventElapsedTime(&a, ev[4 * i], ev[4 * i + 1]));
      TPO_CK(cudaEventElapsedTime(&b, ev[4 * i + 2], ev[4 * i + 3]));
      g_prof.dir_ms += a;
      g_prof.update_ms += b;
    }
    if (real > 0 && lb.step == 0) {
      g_prof.dir_launches += real;
      g_prof.update_launches += real;
      g_prof.dir_bytes += (int64_t)real * lb.dir;
      g_prof.update_bytes += (int64_t)real * lb.update;
    }
  }
  return TPO_OK;
}

// Algorithmic bytes per launch (compact sizes: N DOFs, E elements, Nn nodes)
template <typename T, int PRE>
LaunchBytes launch_bytes(const tpo_grid *g) {
  const int64_t nn = (int64_t)(g->nelx + 1) * (g->nely + 1), nd = 2 * nn;
  const int64_t ne = (int64_t)g->nelx * g->nely, s = sizeof(T);
  LaunchBytes lb;
  const int64_t su = sizeof(double);  // the solution u is FP64 in both forms
  lb.dir = 4 * nd * s + ne * s + nn;  // r|z, p_old -> p, Ap; scales; mask
  if (PRE == TPO_PRECOND_BLOCK_JACOBI)
    lb.update = 5 * nd * s + 2 * nd * su + ne * s + nn;  // r, Ap, p, u -> u, r', z; weights
  else  // u, r, p, Ap -> u, r, z
    lb.update = 5 * nd * s + 2 * nd * su + (PRE == TPO_PRECOND_NONE ? 0 : ne * s) + nn;
  return lb;
}

// one-launch iteration: r, w, s, p, x read and written, scales, mask
template <typename T>
LaunchBytes step_bytes(const tpo_grid *g) {
  const int64_t nn = (int64_t)(g->nelx + 1) * (g->nely + 1), nd = 2 * nn;
  const int64_t ne = (int64_t)g->nelx * g->nely, s = sizeof(T);
  LaunchBytes lb{0, 0, 10 * nd * s + ne * s + nn};
  return lb;
}

int pack_inputs(const tpo_grid *g, const PcgWs &w, const double *f, const uint8_t *fixed,
                const double *u, bool warm, cudaStream_t st) {
  const int nx = g->nelx, ny = g->nely, P = w.P;
  const size_t NN = (size_t)(nx + 1) * P;
  const dim3 fg = flat_grid(NN, 256, sm_count() * 16);
  k_pack_mask<<<fg, 256, 0, st>>>(nx, ny, P, fixed, w.mask);
  TPO_CK_LAUNCH();
  k_pack_nodes<double><<<fg, 256, 0, st>>>(nx, ny, P, f, w.f);
  TPO_CK_LAUNCH();
  if (warm) {
    k_pack_nodes<double><<<fg, 256, 0, st>>>(nx, ny, P, u, w.u);
    TPO_CK_LAUNCH();
  } else {
    TPO_CK(cudaMemsetAsync(w.u, 0, 2 * NN * sizeof(double), st));
  }
  return TPO_OK;
}

// Zero every PCG vector once per solve: the kernels write only grid rows, so
// the pad slots (which the stencils read as zero neighbours) stay zero.
int zero_vectors(const PcgWs &w, size_t NN, cudaStream_t st) {
  double *d64[] = {w.ra, w.rb, w.pa, w.pb, w.ap, w.z, w.wa, w.wb, w.sa, w.sb};
  for (double *p : d64)
    if (p) TPO_CK(cudaMemsetAsync(p, 0, 2 * NN * sizeof(double), st));
  float *d32[] = {w.fra, w.frb, w.fpa, w.fpb, w.fap, w.fz};
  for (float *p : d32)
    if (p) TPO_CK(cudaMemsetAsync(p, 0, 2 * NN * sizeof(float), st));
  return TPO_OK;
}

int unpack_solution(const tpo_grid *g, const PcgWs &w, double *u, cudaStream_t st) {
  const size_t n = (size_t)(g->nelx + 1) * (g->nely + 1);
  k_unpack_nodes<<<flat_grid(n, 256, sm_count() * 16), 256, 0, st>>>(g->nelx, g->nely, w.P, w.u,
                                                                      u);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// ----------------------------------------------------------------- FP64 PCG
template <int PRE>
int pcg_fp64(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho, const double *f,
             const uint8_t *fixed, double *u, const PcgWs &w, tpo_solve_result *out,
             cudaStream_t st, double alpha_reg) {
  const int nx = g->nelx, ny = g->nely, P = w.P;
  constexpr bool block = PRE == TPO_PRECOND_BLOCK_JACOBI;
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);
  int rc = pack_inputs(g, w, f, fixed, u, c->warm_start != 0, st);
  if (rc) return rc;
  if ((rc = zero_vectors(w, (size_t)(nx + 1) * P, st))) return rc;
  k_scales<<<flat_grid((size_t)nx * P, 256, sm_count() * 16), 256, 0, st>>>(
      nx, ny, P, rho, g->e_min, g->penalty, alpha_reg, w.s64, nullptr, block ? w.w64 : nullptr,
      nullptr);
  TPO_CK_LAUNCH();
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, 0.0, c->max_iter, nullptr, 0.0, 0);
  TPO_CK_LAUNCH();

  TsArgs a{};
  a.nx = nx;
  a.ny = ny;
  a.P = P;
  a.s = w.s64;
  a.mask = w.mask;
  a.a = w.u;
  a.uw = w.u;
  a.f = w.f;
  a.out = w.ra;
  a.part = w.part;
  a.ctl = w.ctl;
  a.err = &w.ctl->err;
  StencilCfg<double, double, M_RES, PRE>::launch(st, a, nx, ny);
  TPO_CK_LAUNCH();

  BlkArgs b{};
  b.nx = nx;
  b.ny = ny;
  b.P = P;
  b.w = w.w64;
  b.mask = w.mask;
  b.u = w.u;
  b.ap = w.ap;
  b.pa = w.pa;
  b.pb = w.pb;
  b.ra = w.ra;
  b.rb = w.rb;
  b.z = w.z;
  b.part = w.part;
  b.ctl = w.ctl;
  if (block) {
    k_blockpre<double, double, true, kBlkL><<<blk_grid(nx, ny), ST_THREADS, 0, st>>>(b);
    TPO_CK_LAUNCH();
  } else {
    k_precond_flat<double, double, PRE><<<flat_wave<k_precond_flat<double, double, PRE>>(nx, ny),
                                            UF_THREADS, 0, st>>>(
        nx, ny, P, w.s64, w.mask, w.ra, w.z);
    TPO_CK_LAUNCH();
  }

  TsArgs d{};
  d.nx = nx;
  d.ny = ny;
  d.P = P;
  d.s = w.s64;
  d.mask = w.mask;
  d.a = w.z;  // z from the update kernel (or the element-block preconditioner)
  d.pa = w.pa;
  d.pb = w.pb;
  d.out = w.ap;
  d.part = w.part;
  d.ctl = w.ctl;
  d.err = &w.ctl->err;
  UpdArgs up{};
  up.nx = nx;
  up.ny = ny;
  up.P = P;
  up.s = w.s64;
  up.mask = w.mask;
  up.u = w.u;
  up.r = w.ra;
  up.ap = w.ap;
  up.pa = w.pa;
  up.pb = w.pb;
  up.part = w.part;
  up.ctl = w.ctl;
  up.z = w.z;

  auto iter = [&](cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    StencilCfg<double, double, M_DIR, TPO_PRECOND_BLOCK_JACOBI>::launch(st, d, nx, ny);  // reads z
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    if (ev) TPO_CK(cudaEventRecord(ev[2], st));
    if (block) {
      k_blockpre<double, double, false, kBlkL><<<blk_grid(nx, ny), ST_THREADS, 0, st>>>(b);
    } else {
      k_update_flat<double, double, PRE>
          <<<flat_wave<k_update_flat<double, double, PRE>>(nx, ny), UF_THREADS, 0, st>>>(up);
    }
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[3], st));
    return TPO_OK;
  };
  PcgCtl fin;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  rc = run_iterations(iter, w.ctl, c->max_iter, 0, chunk, st, &fin, launch_bytes<double, PRE>(g));
  if (rc) return rc;
  if ((rc = unpack_solution(g, w, u, st))) return rc;
  TPO_CK(cudaStreamSynchronize(st));
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
// One PCG whose Krylov vectors (r, p, Ap, z) are stored in FP32, with FP64
// arithmetic, dot products and solution u. Its recursive residual is replaced
// by the true FP64 residual f - K u whenever it has dropped by inner_tol since
// the last replacement ("reliable updates"); the search direction is kept
// across replacements, so the Krylov space is not discarded. Convergence is
// decided only on the FP64 residual.
template <int PRE>
int pcg_mixed(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho, const double *f,
              const uint8_t *fixed, double *u, const PcgWs &w, tpo_solve_result *out,
              cudaStream_t st, double alpha_reg) {
  const int nx = g->nelx, ny = g->nely, P = w.P;
  const size_t NN = (size_t)(nx + 1) * P;
  constexpr bool block = PRE == TPO_PRECOND_BLOCK_JACOBI;
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);
  const double delta = c->inner_tol > 0.0 ? c->inner_tol : 1e-3;
  int rc = pack_inputs(g, w, f, fixed, u, c->warm_start != 0, st);
  if (rc) return rc;
  if ((rc = zero_vectors(w, NN, st))) return rc;
  k_scales<<<flat_grid((size_t)nx * P, 256, sm_count() * 16), 256, 0, st>>>(
      nx, ny, P, rho, g->e_min, g->penalty, alpha_reg, w.s64, w.s32, nullptr,
      block ? w.w32 : nullptr);
  TPO_CK_LAUNCH();
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, delta * delta, c->max_iter, w.octl, tol_sq,
                              c->max_outer);
  TPO_CK_LAUNCH();

  TsArgs rx{};
  rx.nx = nx;
  rx.ny = ny;
  rx.P = P;
  rx.s = w.s64;
  rx.mask = w.mask;
  rx.a = w.u;
  rx.uw = w.u;
  rx.f = w.f;
  rx.part = w.part;
  rx.ctl = w.ctl;
  rx.octl = w.octl;
  rx.err = &w.ctl->err;

  BlkArgs b{};
  b.nx = nx;
  b.ny = ny;
  b.P = P;
  b.w = w.w32;
  b.mask = w.mask;
  b.u = w.u;
  b.ap = w.fap;
  b.pa = w.fpa;
  b.pb = w.fpb;
  b.ra = w.fra;
  b.rb = w.frb;
  b.z = w.fz;
  b.part = w.part;
  b.ctl = w.ctl;

  TsArgs d{};
  d.nx = nx;
  d.ny = ny;
  d.P = P;
  d.s = w.s32;
  d.mask = w.mask;
  d.a = w.fz;  // z from the update kernel (or the element-block preconditioner)
  d.pa = w.fpa;
  d.pb = w.fpb;
  d.out = w.fap;
  d.part = w.part;
  d.ctl = w.ctl;
  d.err = &w.ctl->err;
  UpdArgs up{};
  up.nx = nx;
  up.ny = ny;
  up.P = P;
  up.s = w.s32;
  up.mask = w.mask;
  up.u = w.u;
  up.r = w.fra;
  up.ap = w.fap;
  up.pa = w.fpa;
  up.pb = w.fpb;
  up.part = w.part;
  up.ctl = w.ctl;
  up.z = w.fz;

  auto iter = [&](cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    StencilCfg<float, double, M_DIR, TPO_PRECOND_BLOCK_JACOBI>::launch(st, d, nx, ny);  // reads z
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    if (ev) TPO_CK(cudaEventRecord(ev[2], st));
    if (block) {
      k_blockpre<float, double, false, kBlkL, double>
          <<<blk_grid(nx, ny), ST_THREADS, 0, st>>>(b);
    } else {
      k_update_flat<float, double, PRE, double>
          <<<flat_wave<k_update_flat<float, double, PRE, double>>(nx, ny), UF_THREADS, 0, st>>>(up);
    }
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[3], st));
    return TPO_OK;
  };

  Poller *pl;
  if ((rc = get_poller(&pl))) return rc;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  OuterCtl oh{};
  PcgCtl fin{};
  int status = TPO_SOLVE_MAX_ITER, inner_it = 0;
  for (int k = 0;; ++k) {
    // block preconditioner: the current residual buffer follows the iteration parity
    rx.out = (block && (inner_it & 1)) ? (void *)w.frb : (void *)w.fra;
    StencilCfg<double, double, M_RESX, PRE>::launch(st, rx, nx, ny);
    TPO_CK_LAUNCH();
    if (block) {
      k_blockpre<float, double, true, kBlkL, double>
          <<<blk_grid(nx, ny), ST_THREADS, 0, st>>>(b);
      TPO_CK_LAUNCH();
    } else {  // z of the replaced residual (no-op when the replacement did not run)
      k_precond_flat<float, double, PRE><<<flat_wave<k_precond_flat<float, double, PRE>>(nx, ny),
                                          UF_THREADS, 0, st>>>(
          nx, ny, P, w.s32, w.mask, w.fra, w.fz);
      TPO_CK_LAUNCH();
    }
    int err = 0;  // a pipeline wait of the residual kernels ran out
    TPO_CK(cudaMemcpyAsync(&oh, w.octl, sizeof(OuterCtl), cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaMemcpyAsync(&err, &w.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaStreamSynchronize(st));
    if (err) return fail(TPO_ERR_TIMEOUT, "a TMA pipeline wait ran out of time");
    if (oh.status != TPO_SOLVE_RUNNING) {
      status = oh.status;
      break;
    }
    if (k > 0 && fin.status != SOLVE_NEED_UPDATE) {
      status = fin.status;  // inner solve stopped (max_iter, breakdown): report it
      break;
    }
    if (oh.it > c->max_outer) {
      status = TPO_SOLVE_MAX_ITER;
      break;
    }
    rc = run_iterations(iter, w.ctl, c->max_iter, inner_it, chunk, st, &fin,
                        launch_bytes<float, PRE>(g));
    if (rc) return rc;
    inner_it = fin.it;
    if (fin.status == TPO_SOLVE_NONFINITE) {
      status = TPO_SOLVE_NONFINITE;
      break;
    }
    if (fin.status == TPO_SOLVE_RUNNING) fin.status = TPO_SOLVE_MAX_ITER;
  }
  if ((rc = unpack_solution(g, w, u, st))) return rc;
  TPO_CK(cudaStreamSynchronize(st));
  out->status = status;
  out->iters = inner_it;
  out->updates = inner_it;
  out->outer_iters = oh.it;
  out->rr = oh.rr;
  return TPO_OK;
}

// ----------------------------------------------------------------- one-launch PCG
CgArgs cg_args(const tpo_grid *g, const PcgWs &w) {
  CgArgs a{};
  a.nx = g->nelx;
  a.ny = g->nely;
  a.P = w.P;
  a.mask = w.mask;
  a.s = w.s64;
  a.ra = w.ra;
  a.rb = w.rb;
  a.wa = w.wa;
  a.wb = w.wb;
  a.sa = w.sa;
  a.sb = w.sb;
  a.p = w.pa;
  a.x = w.u;
  a.part = w.part;
  a.ctl = w.ctl;
  a.err = &w.ctl->err;
  return a;
}

// Plain FP64: r = f - K u, the INIT launch, then one launch per iteration.
template <int PRE>
int pcg_single(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho, const double *f,
               const uint8_t *fixed, double *u, const PcgWs &w, tpo_solve_result *out,
               cudaStream_t st, double alpha_reg) {
  const int nx = g->nelx, ny = g->nely, P = w.P;
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);
  int rc = pack_inputs(g, w, f, fixed, u, c->warm_start != 0, st);
  if (rc) return rc;
  if ((rc = zero_vectors(w, (size_t)(nx + 1) * P, st))) return rc;
  k_scales<<<flat_grid((size_t)nx * P, 256, sm_count() * 16), 256, 0, st>>>(
      nx, ny, P, rho, g->e_min, g->penalty, alpha_reg, w.s64, nullptr, nullptr, nullptr);
  TPO_CK_LAUNCH();
  k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, 0.0, c->max_iter, nullptr, 0.0, 0);
  TPO_CK_LAUNCH();

  TsArgs a{};
  a.nx = nx;
  a.ny = ny;
  a.P = P;
  a.s = w.s64;
  a.mask = w.mask;
  a.a = w.u;
  a.uw = w.u;
  a.f = w.f;
  a.out = w.ra;  // phase 0 reads ra
  a.part = w.part;
  a.ctl = w.ctl;
  a.err = &w.ctl->err;
  StencilCfg<double, double, M_RES, PRE>::launch(st, a, nx, ny);
  TPO_CK_LAUNCH();

  const CgArgs ca = cg_args(g, w);
  CgCfg<double, double, PRE>::launch(st, ca, nx, ny);  // INIT
  TPO_CK_LAUNCH();
  auto iter = [&](cudaEvent_t *ev) -> int {
    if (ev) TPO_CK(cudaEventRecord(ev[0], st));
    CgCfg<double, double, PRE>::launch(st, ca, nx, ny);
    TPO_CK_LAUNCH();
    if (ev) TPO_CK(cudaEventRecord(ev[1], st));
    return TPO_OK;
  };
  PcgCtl fin;
  const int chunk = c->poll_every > 0 ? c->poll_every : 16;
  rc = run_iterations(iter, w.ctl, c->max_iter, 0, chunk, st, &fin, step_bytes<double>(g));
  if (rc) return rc;
  if ((rc = unpack_solution(g, w, u, st))) return rc;
  TPO_CK(cudaStreamSynchronize(st));
  int status = fin.status;
  if (status == TPO_SOLVE_RUNNING) status = TPO_SOLVE_MAX_ITER;  // max_iter <= 0
  out->status = status;
  out->updates = fin.it;
  out->iters = (status == TPO_SOLVE_CONVERGED) ? fin.it : c->max_iter;
  out->outer_iters = 1;
  out->rr = fin.rr;
  return TPO_OK;
}

// ----------------------------------------------------------------- asynchronous PCG
// tpo_pcg_solve_async: the same solve as tpo_pcg_solve, enqueued on the stream
// with no host synchronisation. The PCG loop is a CUDA graph conditional
// WHILE node whose body holds kAsyncBody iterations; after each body one
// thread decides on the device whether another is needed (the stop rules are
// the kernels' own; a body limit bounds the loop). A last kernel writes the
// tpo_solve_result into device memory.
constexpr int kAsyncBody = 16;

__global__ void k_solve_cond(const PcgCtl *ctl, const OuterCtl *octl, uint32_t *bodies,
                             uint32_t max_bodies, cudaGraphConditionalHandle h) {
  bool more;
  if (octl)  // mixed: the outer solve runs; the inner one runs or awaits a replacement
    more = octl->status == TPO_SOLVE_RUNNING &&
           (ctl->status == TPO_SOLVE_RUNNING || ctl->status == SOLVE_NEED_UPDATE);
  else
    more = ctl->status == TPO_SOLVE_RUNNING;
  if (ctl->err) more = false;
  const uint32_t b = ++*bodies;
  if (b >= max_bodies) more = false;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

// The host epilogues of pcg_fp64 / pcg_single / pcg_mixed, on the device.
__global__ void k_solve_result(const PcgCtl *ctl, const OuterCtl *octl, const uint32_t *bodies,
                               uint32_t max_bodies, int max_iter, int n_fixed, int n_body,
                               tpo_solve_result *out) {
  int status;
  tpo_solve_result r{};
  if (octl) {
    if (octl->status != TPO_SOLVE_RUNNING) status = octl->status;
    else if (ctl->status != TPO_SOLVE_RUNNING && ctl->status != SOLVE_NEED_UPDATE)
      status = ctl->status;  // the inner solve stopped (max_iter, breakdown, non-finite)
    else
      status = TPO_SOLVE_MAX_ITER;
    r.iters = ctl->it;
    r.updates = ctl->it;
    r.outer_iters = octl->it;
    r.rr = octl->rr;
  } else {
    status = ctl->status;
    if (status == TPO_SOLVE_RUNNING) status = TPO_SOLVE_MAX_ITER;
    r.updates = ctl->it;
    r.iters = status == TPO_SOLVE_CONVERGED ? ctl->it : max_iter;
    r.outer_iters = 1;
    r.rr = ctl->rr;
  }
  if (ctl->err) status = TPO_SOLVE_TIMEOUT;
  else if (*bodies >= max_bodies && (status == TPO_SOLVE_MAX_ITER) &&
           (octl ? octl->status == TPO_SOLVE_RUNNING : ctl->status == TPO_SOLVE_RUNNING))
    status = TPO_SOLVE_LOOP_LIMIT;
  r.status = status;
  r.bodies = (int32_t)*bodies;
  r.launches = n_fixed + (int32_t)*bodies * n_body;
  *out = r;
}

__global__ void k_solve_zero_rhs(tpo_solve_result *out) {
  tpo_solve_result r{};
  r.status = TPO_SOLVE_ZERO_RHS;
  r.outer_iters = 1;
  r.launches = 1;
  *out = r;
}

// two private non-blocking streams per device: one into which the loop body
// is captured, one into which a solve is captured when the caller's stream is
// not capturing (the caller's stream may be the legacy default stream, which
// cannot be captured; the finished graph is launched on it instead)
cudaStream_t g_body_stream[kMaxDevices], g_cap_stream[kMaxDevices];
std::mutex g_body_mu;
int capture_streams(cudaStream_t *body, cudaStream_t *cap) {
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_body_mu);
  if (!g_body_stream[dev])
    TPO_CK(cudaStreamCreateWithFlags(&g_body_stream[dev], cudaStreamNonBlocking));
  if (!g_cap_stream[dev])
    TPO_CK(cudaStreamCreateWithFlags(&g_cap_stream[dev], cudaStreamNonBlocking));
  if (body) *body = g_body_stream[dev];
  if (cap) *cap = g_cap_stream[dev];
  return TPO_OK;
}

// Inserts the loop into the capture that `st` is running: a WHILE node after
// the work captured so far, its body captured from `emit(body_stream)`, and
// the stream's later work ordered after the node.
template <typename BodyFn>
int add_while_loop(cudaStream_t st, BodyFn emit, const PcgCtl *ctl, const OuterCtl *octl,
                   uint32_t *bodies, uint32_t max_bodies, int *n_body) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  TPO_CK(cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, &deps, &ndeps));
  if (cst != cudaStreamCaptureStatusActive || !g)
    return fail(TPO_ERR_CUDA, "the stream is not capturing");
  std::vector<cudaGraphNode_t> pre(deps, deps + ndeps);
  cudaGraphConditionalHandle h;
  TPO_CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  TPO_CK(cudaGraphAddNode(&cnode, g, pre.data(), pre.size(), &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t bs;
  int rc = capture_streams(&bs, nullptr);
  if (rc) return rc;
  TPO_CK(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed));
  const int64_t l0 = g_launches.load();
  rc = emit(bs);
  *n_body = (int)(g_launches.load() - l0) + 1;  // + the condition kernel
  if (!rc) {
    k_solve_cond<<<1, 1, 0, bs>>>(ctl, octl, bodies, max_bodies, h);
    if (cudaPeekAtLastError() != cudaSuccess) rc = fail(TPO_ERR_CUDA, "loop condition launch");
  }
  cudaGraph_t tmp;
  const cudaError_t e = cudaStreamEndCapture(bs, &tmp);
  if (rc) return rc;
  TPO_CK(e);
  TPO_CK(cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies));
  return TPO_OK;
}

// The whole solve of one form enqueued on `st`, which is capturing: the
// set-up of pcg_mixed / pcg_single / pcg_fp64, the loop, the epilogue. Same
// kernels in the same order as the host-driven solve, so the same results.
template <int PRE>
int emit_solve_async(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho,
                     const double *f, const uint8_t *fixed, double *u, const PcgWs &w,
                     tpo_solve_result *out, cudaStream_t st, double alpha_reg) {
  const int nx = g->nelx, ny = g->nely, P = w.P;
  const size_t NN = (size_t)(nx + 1) * P;
  constexpr bool block = PRE == TPO_PRECOND_BLOCK_JACOBI;
  const bool mixed = c->precision == TPO_PRECISION_MIXED;
  const double fn = std::sqrt(c->f_norm_sq);
  const double tol_sq = (c->tol * fn) * (c->tol * fn);
  const dim3 sg = flat_grid((size_t)nx * P, 256, sm_count() * 16);
  const int64_t l0 = g_launches.load();
  int n_body = 0;
  int rc = pack_inputs(g, w, f, fixed, u, c->warm_start != 0, st);
  if (rc) return rc;
  if ((rc = zero_vectors(w, NN, st))) return rc;
  TPO_CK(cudaMemsetAsync(w.bodies, 0, sizeof(uint32_t), st));
  constexpr int m = kAsyncBody;
  uint32_t max_bodies = 0;
  if (mixed) {
    k_scales<<<sg, 256, 0, st>>>(nx, ny, P, rho, g->e_min, g->penalty, alpha_reg, w.s64, w.s32,
                                 nullptr, block ? w.w32 : nullptr);
    TPO_CK_LAUNCH();
    const double delta = c->inner_tol > 0.0 ? c->inner_tol : 1e-3;
    k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, delta * delta, c->max_iter, w.octl, tol_sq,
                                c->max_outer);
    TPO_CK_LAUNCH();
    TsArgs rx{};
    rx.nx = nx; rx.ny = ny; rx.P = P;
    rx.s = w.s64; rx.mask = w.mask; rx.a = w.u; rx.uw = w.u; rx.f = w.f;
    rx.out = w.fra; rx.out2 = block ? w.frb : nullptr;  // block: by iteration parity
    rx.part = w.part; rx.ctl = w.ctl; rx.octl = w.octl; rx.err = &w.ctl->err;
    BlkArgs b{};
    b.nx = nx; b.ny = ny; b.P = P;
    b.w = w.w32; b.mask = w.mask; b.u = w.u; b.ap = w.fap; b.pa = w.fpa; b.pb = w.fpb;
    b.ra = w.fra; b.rb = w.frb; b.z = w.fz; b.part = w.part; b.ctl = w.ctl;
    TsArgs d{};
    d.nx = nx; d.ny = ny; d.P = P;
    d.s = w.s32; d.mask = w.mask; d.a = w.fz; d.pa = w.fpa; d.pb = w.fpb; d.out = w.fap;
    d.part = w.part; d.ctl = w.ctl; d.err = &w.ctl->err;
    UpdArgs up{};
    up.nx = nx; up.ny = ny; up.P = P;
    up.s = w.s32; up.mask = w.mask; up.u = w.u; up.r = w.fra; up.ap = w.fap; up.pa = w.fpa;
    up.pb = w.fpb; up.part = w.part; up.ctl = w.ctl; up.z = w.fz;
    // a body: the FP64 residual replacement (a no-op unless one is due), z of
    // a replaced residual, then m inner iterations (no-ops once one is due)
    max_bodies = (uint32_t)((c->max_iter + m - 1) / m + c->max_outer + 2);
    auto body = [&](cudaStream_t bs) -> int {
      StencilCfg<double, double, M_RESX, PRE>::launch(bs, rx, nx, ny);
      TPO_CK_LAUNCH();
      if (block) {
        BlkArgs bi = b;
        bi.gate = 1;
        k_blockpre<float, double, true, kBlkL, double><<<blk_grid(nx, ny), ST_THREADS, 0, bs>>>(bi);
      } else {
        k_precond_gated<float, double, PRE>
            <<<flat_wave<k_precond_gated<float, double, PRE>>(nx, ny), UF_THREADS, 0, bs>>>(
                w.ctl, nx, ny, P, w.s32, w.mask, w.fra, w.fz);
      }
      TPO_CK_LAUNCH();
      for (int i = 0; i < m; ++i) {
        StencilCfg<float, double, M_DIR, TPO_PRECOND_BLOCK_JACOBI>::launch(bs, d, nx, ny);
        TPO_CK_LAUNCH();
        if (block)
          k_blockpre<float, double, false, kBlkL, double><<<blk_grid(nx, ny), ST_THREADS, 0, bs>>>(b);
        else
          k_update_flat<float, double, PRE, double>
              <<<flat_wave<k_update_flat<float, double, PRE, double>>(nx, ny), UF_THREADS, 0, bs>>>(up);
        TPO_CK_LAUNCH();
      }
      return TPO_OK;
    };
    rc = add_while_loop(st, body, w.ctl, w.octl, w.bodies, max_bodies, &n_body);
  } else {
    k_scales<<<sg, 256, 0, st>>>(nx, ny, P, rho, g->e_min, g->penalty, alpha_reg, w.s64, nullptr,
                                 block ? w.w64 : nullptr, nullptr);
    TPO_CK_LAUNCH();
    k_ctl_init<<<1, 1, 0, st>>>(w.ctl, tol_sq, 0.0, c->max_iter, nullptr, 0.0, 0);
    TPO_CK_LAUNCH();
    TsArgs a{};
    a.nx = nx; a.ny = ny; a.P = P;
    a.s = w.s64; a.mask = w.mask; a.a = w.u; a.uw = w.u; a.f = w.f; a.out = w.ra;
    a.part = w.part; a.ctl = w.ctl; a.err = &w.ctl->err;
    StencilCfg<double, double, M_RES, PRE>::launch(st, a, nx, ny);
    TPO_CK_LAUNCH();
    if (w.single) {
      const CgArgs ca = cg_args(g, w);
      // the first launch of the first body is the INIT launch
      max_bodies = (uint32_t)((c->max_iter + 1 + m - 1) / m + 2);
      auto body = [&](cudaStream_t bs) -> int {
        for (int i = 0; i < m; ++i) {
          CgCfg<double, double, PRE>::launch(bs, ca, nx, ny);
          TPO_CK_LAUNCH();
        }
        return TPO_OK;
      };
      rc = add_while_loop(st, body, w.ctl, nullptr, w.bodies, max_bodies, &n_body);
    } else {
      BlkArgs b{};
      b.nx = nx; b.ny = ny; b.P = P;
      b.w = w.w64; b.mask = w.mask; b.u = w.u; b.ap = w.ap; b.pa = w.pa; b.pb = w.pb;
      b.ra = w.ra; b.rb = w.rb; b.z = w.z; b.part = w.part; b.ctl = w.ctl;
      if (block) {
        k_blockpre<double, double, true, kBlkL><<<blk_grid(nx, ny), ST_THREADS, 0, st>>>(b);
      } else {
        k_precond_flat<double, double, PRE>
            <<<flat_wave<k_precond_flat<double, double, PRE>>(nx, ny), UF_THREADS, 0, st>>>(
                nx, ny, P, w.s64, w.mask, w.ra, w.z);
      }
      TPO_CK_LAUNCH();
      TsArgs d{};
      d.nx = nx; d.ny = ny; d.P = P;
      d.s = w.s64; d.mask = w.mask; d.a = w.z; d.pa = w.pa; d.pb = w.pb; d.out = w.ap;
      d.part = w.part; d.ctl = w.ctl; d.err = &w.ctl->err;
      UpdArgs up{};
      up.nx = nx; up.ny = ny; up.P = P;
      up.s = w.s64; up.mask = w.mask; up.u = w.u; up.r = w.ra; up.ap = w.ap; up.pa = w.pa;
      up.pb = w.pb; up.part = w.part; up.ctl = w.ctl; up.z = w.z;
      max_bodies = (uint32_t)((c->max_iter + m - 1) / m + 2);
      auto body = [&](cudaStream_t bs) -> int {
        for (int i = 0; i < m; ++i) {
          StencilCfg<double, double, M_DIR, TPO_PRECOND_BLOCK_JACOBI>::launch(bs, d, nx, ny);
          TPO_CK_LAUNCH();
          if (block)
            k_blockpre<double, double, false, kBlkL><<<blk_grid(nx, ny), ST_THREADS, 0, bs>>>(b);
          else
            k_update_flat<double, double, PRE>
                <<<flat_wave<k_update_flat<double, double, PRE>>(nx, ny), UF_THREADS, 0, bs>>>(up);
          TPO_CK_LAUNCH();
        }
        return TPO_OK;
      };
      rc = add_while_loop(st, body, w.ctl, nullptr, w.bodies, max_bodies, &n_body);
    }
  }
  if (rc) return rc;
  if ((rc = unpack_solution(g, w, u, st))) return rc;
  // kernels outside the loop: those enqueued so far less one body's, plus this one
  const int n_fixed = (int)(g_launches.load() - l0) - (n_body - 1) + 1;
  k_solve_result<<<1, 1, 0, st>>>(w.ctl, mixed ? w.octl : nullptr, w.bodies, max_bodies,
                                  c->max_iter, n_fixed, n_body, out);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

}  // namespace

// ------------------------------------------------------------------ matvec (packing)
template <typename T, typename C>
static int apply_impl(const tpo_grid *g, const T *elem, bool from_density, const uint8_t *fixed,
                      const T *p, T *ap, double *pap_out, void *ws, size_t ws_bytes,
                      tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!elem || !fixed || !p || !ap || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(p, 2 * sizeof(T)) || !aligned(ap, 2 * sizeof(T)) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer");
  if (ws_bytes < tpo_matvec_workspace_bytes(g))
    return fail(TPO_ERR_WORKSPACE, "workspace too small");
  const int nx = g->nelx, ny = g->nely, P = pad_pitch(ny);
  const size_t NN = (size_t)(nx + 1) * P, NE = (size_t)nx * P;
  cudaStream_t st = static_cast<cudaStream_t>(s);
  Carve cv(ws);
  PcgCtl *ctl = cv.take<PcgCtl>(1);
  double *part = cv.take<double>((size_t)max_ctas(g));
  uint8_t *mask = cv.take<uint8_t>(NN);
  T *sc = cv.take<T>(NE);
  T *pp = cv.take<T>(2 * NN);
  T *app = cv.take<T>(2 * NN);
  const dim3 fg = flat_grid(NN, 256, sm_count() * 16);
  TPO_CK(cudaMemsetAsync(ctl, 0, sizeof(PcgCtl), st));
  if (from_density)
    k_scales_t<T><<<flat_grid(NE, 256, sm_count() * 16), 256, 0, st>>>(nx, ny, P, elem, g->e_min,
                                                                       g->penalty, sc);
  else
    k_pad_elems<T><<<flat_grid(NE, 256, sm_count() * 16), 256, 0, st>>>(nx, ny, P, elem, sc);
  TPO_CK_LAUNCH();
  k_pack_mask<<<fg, 256, 0, st>>>(nx, ny, P, fixed, mask);
  TPO_CK_LAUNCH();
  k_pack_nodes_t<T><<<fg, 256, 0, st>>>(nx, ny, P, p, pp);
  TPO_CK_LAUNCH();
  TsArgs a{};
  a.nx = nx;
  a.ny = ny;
  a.P = P;
  a.s = sc;
  a.mask = mask;
  a.a = pp;
  a.out = app;
  a.part = part;
  a.ctl = ctl;
  a.result = pap_out;
  a.err = &ctl->err;
  cudaEvent_t *ev = nullptr;
  if (g_prof_on && (rc = prof_events(1, &ev))) return rc;
  if (ev) TPO_CK(cudaEventRecord(ev[0], st));
  StencilCfg<T, C, M_RAW, TPO_PRECOND_NONE>::launch(st, a, nx, ny);
  TPO_CK_LAUNCH();
  if (ev) {
    TPO_CK(cudaEventRecord(ev[1], st));
    TPO_CK(cudaEventSynchronize(ev[1]));
    float ms = 0.f;
    TPO_CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    const int64_t nn = (int64_t)(nx + 1) * (ny + 1);
    g_prof.apply_launches += 1;
    g_prof.apply_ms += ms;
    g_prof.apply_bytes += 4 * nn * (int64_t)sizeof(T) + (int64_t)nx * ny * sizeof(T) + nn;
  }
  k_unpack_nodes_t<T><<<flat_grid((size_t)(nx + 1) * (ny + 1), 256, sm_count() * 16), 256, 0,
                        st>>>(nx, ny, P, app, ap);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

// =================================================================== C ABI
extern "C" {

int tpo_version(void) { return 1; }

int tpo_test_withhold_stage(int32_t group) {
  if (group < 0) return fail(TPO_ERR_ARGS, "group must be >= 0");
  g_withhold1.store(group + 1);
  return TPO_OK;
}

const char *tpo_last_error_string(void) { return g_err.c_str(); }

int tpo_set_stiffness(const double ke[64], const double ke_inv[64], double alpha_reg) {
  if (!ke || !ke_inv) return fail(TPO_ERR_ARGS, "ke and ke_inv must be non-NULL");
  int dev;
  int rc = current_device(&dev);
  if (rc) return rc;
  double kst[6];
  rc = stiffness_structure(ke, kst);
  if (rc) return rc;
  float kf[64], kif[64], kstf[6];
  for (int i = 0; i < 64; ++i) {
    kf[i] = (float)ke[i];
    kif[i] = (float)ke_inv[i];
  }
  for (int i = 0; i < 6; ++i) kstf[i] = (float)kst[i];
  TPO_CK(cudaMemcpyToSymbol(c_kst, kst, sizeof(kst)));
  TPO_CK(cudaMemcpyToSymbol(c_kst_f, kstf, sizeof(kstf)));
  TPO_CK(cudaMemcpyToSymbol(c_ke, ke, sizeof(double) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_ke_f, kf, sizeof(float) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_kinv, ke_inv, sizeof(double) * 64));
  TPO_CK(cudaMemcpyToSymbol(c_kinv_f, kif, sizeof(float) * 64));
  g_alpha_reg[dev] = alpha_reg;
  g_have_stiffness[dev] = true;
  // the asynchronous solve's capture streams, made here, outside any capture
  return capture_streams(nullptr, nullptr);
}

// ------------------------------------------------------------------ matvec
size_t tpo_matvec_workspace_bytes(const tpo_grid *g) {
  if (check_grid(g)) return 0;
  const int P = pad_pitch(g->nely);
  const size_t NN = (size_t)(g->nelx + 1) * P, NE = (size_t)g->nelx * P;
  Carve cv(nullptr);
  cv.take<PcgCtl>(1);
  cv.take<double>((size_t)max_ctas(g));
  cv.take<uint8_t>(NN);
  cv.take<double>(NE);
  cv.take<double>(2 * NN);
  cv.take<double>(2 * NN);
  return cv.off;
}

// The FP32 entry points compute in FP32 (the reference's precision); the FP64
// ones in FP64.
int tpo_matvec_f64(const tpo_grid *g, const double *rho, const uint8_t *fixed, const double *p,
                   double *ap, double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  return apply_impl<double, double>(g, rho, true, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_matvec_f32(const tpo_grid *g, const float *rho, const uint8_t *fixed, const float *p,
                   float *ap, double *pap_out, void *ws, size_t ws_bytes, tpo_stream s) {
  return apply_impl<float, float>(g, rho, true, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_apply_stiffness_f64(const tpo_grid *g, const double *scale, const uint8_t *fixed,
                            const double *p, double *ap, double *pap_out, void *ws,
                            size_t ws_bytes, tpo_stream s) {
  return apply_impl<double, double>(g, scale, false, fixed, p, ap, pap_out, ws, ws_bytes, s);
}

int tpo_apply_stiffness_f32(const tpo_grid *g, const float *scale, const uint8_t *fixed,
                            const float *p, float *ap, double *pap_out, void *ws,
                            size_t ws_bytes, tpo_stream s) {
  return apply_impl<float, float>(g, scale, false, fixed, p, ap, pap_out, ws, ws_bytes, s);
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

}  // extern "C"

namespace {
// argument checks shared by tpo_pcg_solve and tpo_pcg_solve_async
int check_solve_args(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho_phys,
                     const double *f, const uint8_t *fixed, double *u, void *ws,
                     size_t ws_bytes, const void *out, int *dev) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!c || !out) return fail(TPO_ERR_ARGS, "cfg and result must be non-NULL");
  if ((rc = need_stiffness(dev))) return rc;
  if (!rho_phys || !f || !fixed || !u || !ws) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(f, 16) || !aligned(u, 16) || !aligned(ws, kAlign))
    return fail(TPO_ERR_ARGS, "misaligned pointer (nodal vectors need 16 B, workspace 256 B)");
  if (c->precond < TPO_PRECOND_NONE || c->precond > TPO_PRECOND_NODAL_BLOCK)
    return fail(TPO_ERR_ARGS, "unknown preconditioner %d", c->precond);
  if (c->precision != TPO_PRECISION_FP64 && c->precision != TPO_PRECISION_MIXED)
    return fail(TPO_ERR_ARGS, "unknown precision %d", c->precision);
  if (c->recurrence < TPO_RECURRENCE_AUTO || c->recurrence > TPO_RECURRENCE_SINGLE)
    return fail(TPO_ERR_ARGS, "unknown recurrence %d", c->recurrence);
  if (c->recurrence == TPO_RECURRENCE_SINGLE &&
      (c->precond == TPO_PRECOND_BLOCK_JACOBI || c->precision != TPO_PRECISION_FP64))
    return fail(TPO_ERR_ARGS,
                "the one-launch recurrence serves the FP64 solve with a point preconditioner "
                "only (not block_jacobi, not the mixed form)");
  if (!(c->tol >= 0.0) || !(c->f_norm_sq >= 0.0))
    return fail(TPO_ERR_ARGS, "tol and f_norm_sq must be >= 0");
  const PcgWs w = carve_pcg(ws, g, c);
  if (ws_bytes < w.bytes) return fail(TPO_ERR_WORKSPACE, "workspace %zu < %zu", ws_bytes, w.bytes);
  return TPO_OK;
}
}  // namespace

extern "C" {

int tpo_pcg_solve(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho_phys,
                  const double *f, const uint8_t *fixed, double *u, void *ws, size_t ws_bytes,
                  tpo_solve_result *out, tpo_stream s) {
  int dev;
  int rc = check_solve_args(g, c, rho_phys, f, fixed, u, ws, ws_bytes, out, &dev);
  if (rc) return rc;
  const PcgWs w = carve_pcg(ws, g, c);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  memset(out, 0, sizeof(*out));

  // reference solver.py:59-63: ||f|| < 1e-30 -> u = 0, no iterations
  if (std::sqrt(c->f_norm_sq) < 1e-30) {
    const size_t nn = (size_t)(g->nelx + 1) * (g->nely + 1);
    TPO_CK(cudaMemsetAsync(u, 0, 2 * nn * sizeof(double), st));
    TPO_CK(cudaStreamSynchronize(st));
    out->status = TPO_SOLVE_ZERO_RHS;
    return TPO_OK;
  }
  const double ar = g_alpha_reg[dev];
  const bool mixed = c->precision == TPO_PRECISION_MIXED;
  const int64_t l0 = g_launches.load();
  auto dispatch = [&]() -> int {
  if (w.single) {
    switch (c->precond) {
      case TPO_PRECOND_NONE:
        return pcg_single<TPO_PRECOND_NONE>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
      case TPO_PRECOND_JACOBI:
        return pcg_single<TPO_PRECOND_JACOBI>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
      default:
        return pcg_single<TPO_PRECOND_NODAL_BLOCK>(g, c, rho_phys, f, fixed, u, w, out, st, ar);
    }
  }
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
  };
  rc = dispatch();
  out->launches = (int32_t)(g_launches.load() - l0);
  return rc;
}

int tpo_pcg_solve_async(const tpo_grid *g, const tpo_solve_cfg *c, const double *rho_phys,
                        const double *f, const uint8_t *fixed, double *u, void *ws,
                        size_t ws_bytes, tpo_solve_result *out_dev, tpo_stream s) {
  int dev;
  int rc = check_solve_args(g, c, rho_phys, f, fixed, u, ws, ws_bytes, out_dev, &dev);
  if (rc) return rc;
  if (!aligned(out_dev, 8)) return fail(TPO_ERR_ARGS, "misaligned result pointer (8 B)");
  const PcgWs w = carve_pcg(ws, g, c);
  const cudaStream_t user = static_cast<cudaStream_t>(s);
  cudaStreamCaptureStatus cs;
  TPO_CK(cudaStreamIsCapturing(user, &cs));
  if (cs == cudaStreamCaptureStatusInvalidated)
    return fail(TPO_ERR_CUDA, "the stream's capture has been invalidated");
  const bool own = cs == cudaStreamCaptureStatusNone;
  cudaStream_t st = user;  // where the solve's nodes are captured
  if (own) {
    if ((rc = capture_streams(nullptr, &st))) return rc;
    TPO_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  }
  const double ar = g_alpha_reg[dev];
  if (std::sqrt(c->f_norm_sq) < 1e-30) {  // reference solver.py:59-63
    const size_t nn = (size_t)(g->nelx + 1) * (g->nely + 1);
    if (cudaMemsetAsync(u, 0, 2 * nn * sizeof(double), st) != cudaSuccess)
      rc = fail(TPO_ERR_CUDA, "memset of u");
    else
      k_solve_zero_rhs<<<1, 1, 0, st>>>(out_dev);
  } else {
    switch (c->precond) {
      case TPO_PRECOND_NONE:
        rc = emit_solve_async<TPO_PRECOND_NONE>(g, c, rho_phys, f, fixed, u, w, out_dev, st, ar);
        break;
      case TPO_PRECOND_JACOBI:
        rc = emit_solve_async<TPO_PRECOND_JACOBI>(g, c, rho_phys, f, fixed, u, w, out_dev, st, ar);
        break;
      case TPO_PRECOND_BLOCK_JACOBI:
        rc = emit_solve_async<TPO_PRECOND_BLOCK_JACOBI>(g, c, rho_phys, f, fixed, u, w, out_dev,
                                                        st, ar);
        break;
      default:
        rc = emit_solve_async<TPO_PRECOND_NODAL_BLOCK>(g, c, rho_phys, f, fixed, u, w, out_dev, st,
                                                       ar);
    }
  }
  if (own) {  // not captured by the caller: run the graph once on the stream
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rc ? rc : fail(TPO_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
    }
    cudaGraphExec_t ex;
    const cudaError_t ei = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    TPO_CK(ei);
    const cudaError_t el = cudaGraphLaunch(ex, user);
    cudaGraphExecDestroy(ex);  // released by the driver once the launch completes
    TPO_CK(el);
  }
  return rc;
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
  if (!aligned(u, 16) || !aligned(ws, kAlign) || !aligned(rho_phys, 8) || !aligned(dc, 8) ||
      !aligned(compliance_out, 8))
    return fail(TPO_ERR_ARGS, "misaligned pointer (u 16 B, doubles 8 B, workspace 256 B)");
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

int tpo_sensitivity_noalloc(const tpo_grid *g, const double *rho_phys, const double *u,
                            double *dc, double *compliance_out, tpo_stream s) {
  int rc = check_grid(g);
  if (rc) return rc;
  int dev;
  if ((rc = need_stiffness(&dev))) return rc;
  if (!rho_phys || !u || !dc || !compliance_out) return fail(TPO_ERR_ARGS, "NULL pointer argument");
  if (!aligned(u, 16) || !aligned(rho_phys, 8) || !aligned(dc, 8) || !aligned(compliance_out, 8))
    return fail(TPO_ERR_ARGS, "misaligned pointer (u 16 B, doubles 8 B)");
  const dim3 gr((g->nely + S_THREADS - 1) / S_THREADS, (g->nelx + SL - 1) / SL, 1);
  const size_t nb = (size_t)gr.x * gr.y;
  if (nb > kSensMaxPartials)
    return fail(TPO_ERR_ARGS,
                "grid %dx%d needs %zu partial sums; the fixed scratch holds %zu "
                "(ceil(nely/128)*ceil(nelx/16) must be <= %zu)",
                g->nelx, g->nely, nb, kSensMaxPartials, kSensMaxPartials);
  // looked up on every call (a host-side query, nothing allocated), so the
  // address always belongs to the device's current context
  void *base = nullptr;
  TPO_CK(cudaGetSymbolAddress(&base, g_sens_scratch));
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

// batched designs (tpo_batch_*): host side, same translation unit
#include "batch_host.cuh"

// 3D (H8) designs (tpo3_*): host side, same translation unit
#include "hex3d_host.cuh"
