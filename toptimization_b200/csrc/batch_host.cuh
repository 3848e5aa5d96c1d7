// Host side of the batched-design engine (tpo_batch_*). Included once, at the
// end of api.cu: it shares that translation unit's error and launch helpers
// and its __constant__ stiffness.
//
// A tpo_batch owns host bookkeeping only (slot table, job tables, CUDA graph);
// every device byte it uses comes from caller workspaces: one for the batch
// (design records, job tables, loop flags) and one per design (its resident
// state), so designs can be admitted and released while others run.
#pragma once

#include "batch.cuh"

struct tpo_batch {
  int dev = 0;
  int max_designs = 0;
  int n_slots = 0;  // slots in use are < n_slots
  tpo_batch_cfg cfg{};
  // device (batch workspace)
  tpo::BDesign *d_designs = nullptr;
  tpo::BJob *d_jobs = nullptr;  // kBK tables of max_designs jobs
  int *d_flag = nullptr;        // [0] loop continues, [1] body limit hit, [2] error word
  unsigned *d_bodies = nullptr;
  int *d_status = nullptr;      // per slot: it, active
  // host mirror
  std::vector<tpo::BDesign> rec;
  std::vector<int> used, h_status;
  int *h_flag = nullptr;        // pinned: 2 poll slots x 4 ints
  cudaEvent_t ev[2]{};
  cudaStream_t cap = nullptr;   // capture stream (graphs cannot be captured on the legacy stream)
  // launch state
  bool dirty = true;
  int njobs[8]{}, nctas[8]{};
  int filter_smem = 0;
  int Ls = 16, Lu = 8;          // strip lengths (columns per CTA) of the stencil / update kinds
  int round_steps = 32;         // PCG steps per round
  cudaGraphExec_t gexec = nullptr;   // OC-iteration graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t rexec = nullptr;   // round graph
  unsigned max_bodies = 0;
};

namespace {

using tpo::BDesign;
using tpo::BJob;

enum BKind { BK_FILTER = 0, BK_SCALES, BK_UNPACK, BK_STENCIL, BK_UPDATE, BK_SENS, kBK };
constexpr int kBatchSteps = 8;       // PCG steps per loop body (one FP64 residual check each)
constexpr int kFlatPerThread = 4;    // elements per thread of the grid-stride kinds

int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

int flat_ctas(int64_t n, int threads) {
  return std::max(1, std::min(4096, cdiv(n, (int64_t)threads * kFlatPerThread)));
}

// per-design launch geometry of each kind (depends on the design and the tiles only)
void kind_geom(int kind, int nx, int ny, int P, int Ls, int Lu, int *gx, int *gy, int *L) {
  *gy = 1;
  *L = 0;
  switch (kind) {
    case BK_FILTER:
      *gx = cdiv(ny, FT);
      *gy = cdiv(nx, FT);
      break;
    case BK_SCALES:
      *gx = flat_ctas((int64_t)nx * P, 256);
      break;
    case BK_UNPACK:
      *gx = flat_ctas((int64_t)(nx + 1) * (ny + 1), 256);
      break;
    case BK_STENCIL:
      *gx = cdiv(ny + 1, RPC);
      *L = Ls;
      *gy = cdiv(nx + 1, Ls);
      break;
    case BK_UPDATE:  // flat grid-stride; Lu = nodes per thread
      *gx = std::max(1, std::min(4096, cdiv((int64_t)(nx + 1) * (ny + 1),
                                            (int64_t)UF_THREADS * Lu)));
      *L = Lu;
      break;
    default:  // BK_SENS
      *gx = cdiv(ny, S_THREADS);
      *gy = cdiv(nx, SL);
      break;
  }
}

constexpr int kMinLs = 8, kMinLu = 4;  // smallest strips: they size the partial-sum buffers

int pcg_part_ctas(int nx, int ny) {
  int gx, gy, L;
  kind_geom(BK_STENCIL, nx, ny, 0, kMinLs, kMinLu, &gx, &gy, &L);
  int m = gx * gy;
  kind_geom(BK_UPDATE, nx, ny, 0, kMinLs, kMinLu, &gx, &gy, &L);
  return std::max(m, gx * gy);
}

struct DesignLayout {
  double *rho, *rho_phys, *dc, *dc_filt, *u, *hist;
  uint8_t *mask;
  double *up, *fp, *s64;
  float *s32, *fr, *fpa, *fpb, *fap, *fz;
  PcgCtl *ctl;
  OuterCtl *octl;
  double *part;
  SumCtl *sc;
  double *spart;
  double *scal;
  size_t bytes;
};

DesignLayout carve_design(void *base, const tpo_batch_design *d) {
  const int nx = d->nelx, ny = d->nely, P = pad_pitch(ny);
  const size_t E = (size_t)nx * ny, Nn = (size_t)(nx + 1) * (ny + 1);
  const size_t NN = (size_t)(nx + 1) * P, NE = (size_t)nx * P;
  Carve cv(base);
  DesignLayout L{};
  L.rho = cv.take<double>(E);
  L.rho_phys = cv.take<double>(E);
  L.dc = cv.take<double>(E);
  L.dc_filt = cv.take<double>(E);
  L.u = cv.take<double>(2 * Nn);
  L.hist = cv.take<double>((size_t)std::max(d->max_oc_iter, 1) * kBatchHist);
  L.mask = cv.take<uint8_t>(NN);
  L.up = cv.take<double>(2 * NN);
  L.fp = cv.take<double>(2 * NN);
  L.s64 = cv.take<double>(NE);
  L.s32 = cv.take<float>(NE);
  L.fr = cv.take<float>(2 * NN);
  L.fpa = cv.take<float>(2 * NN);
  L.fpb = cv.take<float>(2 * NN);
  L.fap = cv.take<float>(2 * NN);
  L.fz = cv.take<float>(2 * NN);
  L.ctl = cv.take<PcgCtl>(1);
  L.octl = cv.take<OuterCtl>(1);
  L.part = cv.take<double>(3 * (size_t)pcg_part_ctas(nx, ny));
  int gx, gy, l;
  L.sc = cv.take<SumCtl>(1);
  kind_geom(BK_SENS, nx, ny, P, kMinLs, kMinLu, &gx, &gy, &l);
  L.spart = cv.take<double>((size_t)gx * gy);
  L.scal = cv.take<double>(8);
  L.bytes = cv.off;
  return L;
}

int check_design(const tpo_batch_design *d) {
  if (!d) return fail(TPO_ERR_ARGS, "design is NULL");
  if (d->nelx < 1 || d->nely < 1) return fail(TPO_ERR_ARGS, "nelx, nely must be >= 1");
  if ((int64_t)(d->nelx + 1) * (d->nely + 1) > (int64_t)1 << 28)
    return fail(TPO_ERR_ARGS, "design too large for a batch slot");
  if (!(d->rmin > 0.0) || (int)std::ceil(d->rmin) > F_MAXR)
    return fail(TPO_ERR_ARGS, "rmin must be in (0, %d]", F_MAXR);
  if (d->max_oc_iter < 1 || d->max_cg_iter < 1 || d->max_outer < 1)
    return fail(TPO_ERR_ARGS, "iteration limits must be >= 1");
  if (!(d->cg_tol > 0.0) || !(d->inner_tol > 0.0) || !(d->f_norm_sq >= 0.0))
    return fail(TPO_ERR_ARGS, "cg_tol, inner_tol must be > 0 and f_norm_sq >= 0");
  return TPO_OK;
}

int filter_smem_bytes(int R) {
  const int W = 2 * R + 1, TW = FT + 2 * R;
  return (W * W + TW * TW) * (int)sizeof(double);
}

template <int PRE> int batch_set_attrs() {
  constexpr int SMEM = TsGeom<double, M_RESX>::template slot_bytes<kBatchG>() * kBatchNG;
  constexpr int SMEM_D = TsGeom<float, M_DIR>::template slot_bytes<kBatchG>() * kBatchNG;
  TPO_CK(cudaFuncSetAttribute(kb_resx<PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
  TPO_CK(cudaFuncSetAttribute(kb_dir<PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_D));
  TPO_CK(cudaFuncSetAttribute(kb_filter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              filter_smem_bytes(F_MAXR)));
  return TPO_OK;
}

// rebuild the job tables of every kind from the active slots
int batch_rebuild(tpo_batch *b, cudaStream_t st) {
  std::vector<BJob> h((size_t)kBK * b->max_designs);
  int maxR = 1;
  unsigned mb = 4;
  for (int k = 0; k < kBK; ++k) {
    int n = 0, cta = 0;
    for (int s = 0; s < b->n_slots; ++s) {
      if (!b->used[s] || !b->h_status[2 * s + 1]) continue;
      const BDesign &D = b->rec[s];
      BJob j{};
      kind_geom(k, D.nx, D.ny, D.P, b->Ls, b->Lu, &j.gx, &j.gy, &j.L);
      j.cta0 = cta;
      j.slot = s;
      cta += j.gx * j.gy;
      h[(size_t)k * b->max_designs + n++] = j;
      if (k == 0) {
        maxR = std::max(maxR, D.R);
        mb = std::max(mb, (unsigned)(D.max_cg + D.max_outer + 4));
      }
    }
    b->njobs[k] = n;
    b->nctas[k] = cta;
  }
  b->filter_smem = filter_smem_bytes(maxR);
  b->max_bodies = mb;
  TPO_CK(cudaMemcpyAsync(b->d_jobs, h.data(), h.size() * sizeof(BJob), cudaMemcpyHostToDevice, st));
  TPO_CK(cudaStreamSynchronize(st));
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (b->rexec) {
    cudaGraphExecDestroy(b->rexec);
    b->rexec = nullptr;
  }
  b->dirty = false;
  return TPO_OK;
}

const BJob *jobs_of(const tpo_batch *b, int kind) {
  return b->d_jobs + (size_t)kind * b->max_designs;
}

// launches of one OC iteration, before and after the PCG loop
int batch_prefix(tpo_batch *b, cudaStream_t st) {
  if (b->nctas[BK_FILTER] == 0) return TPO_OK;
  kb_filter<<<b->nctas[BK_FILTER], F_THREADS, b->filter_smem, st>>>(
      jobs_of(b, BK_FILTER), b->njobs[BK_FILTER], b->d_designs, 0);
  TPO_CK_LAUNCH();
  kb_scales<<<b->nctas[BK_SCALES], 256, 0, st>>>(jobs_of(b, BK_SCALES), b->njobs[BK_SCALES],
                                                  b->d_designs);
  TPO_CK_LAUNCH();
  kb_init<<<cdiv(b->n_slots, 128), 128, 0, st>>>(b->d_designs, b->n_slots);
  TPO_CK_LAUNCH();
  TPO_CK(cudaMemsetAsync(b->d_bodies, 0, sizeof(unsigned), st));
  TPO_CK(cudaMemsetAsync(b->d_flag, 0, 3 * sizeof(int), st));
  return TPO_OK;
}

// RESX, `steps` x (direction, update), then (cond) the loop test
template <int PRE>
int batch_body(tpo_batch *b, cudaStream_t st, cudaGraphConditionalHandle h, int use_h,
               bool cond = true, int steps = kBatchSteps) {
  constexpr int SMEM = TsGeom<double, M_RESX>::template slot_bytes<kBatchG>() * kBatchNG;
  constexpr int SMEM_D = TsGeom<float, M_DIR>::template slot_bytes<kBatchG>() * kBatchNG;
  kb_resx<PRE><<<b->nctas[BK_STENCIL], TS_THREADS, SMEM, st>>>(
      jobs_of(b, BK_STENCIL), b->njobs[BK_STENCIL], b->d_designs);
  TPO_CK_LAUNCH();
  kb_pre<PRE><<<b->nctas[BK_UPDATE], UF_THREADS, 0, st>>>(jobs_of(b, BK_UPDATE),
                                                            b->njobs[BK_UPDATE], b->d_designs);
  TPO_CK_LAUNCH();
  for (int i = 0; i < steps; ++i) {
    kb_dir<PRE><<<b->nctas[BK_STENCIL], TS_THREADS, SMEM_D, st>>>(
        jobs_of(b, BK_STENCIL), b->njobs[BK_STENCIL], b->d_designs, i);
    TPO_CK_LAUNCH();
    kb_update<PRE><<<b->nctas[BK_UPDATE], UF_THREADS, 0, st>>>(
        jobs_of(b, BK_UPDATE), b->njobs[BK_UPDATE], b->d_designs, i);
    TPO_CK_LAUNCH();
  }
  if (!cond) return TPO_OK;
  kb_cond<<<1, 256, 0, st>>>(b->d_designs, b->n_slots, b->d_flag, b->d_bodies, b->max_bodies, h,
                             use_h);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

int batch_suffix(tpo_batch *b, cudaStream_t st) {
  kb_mark<<<cdiv(b->n_slots, 128), 128, 0, st>>>(b->d_designs, b->n_slots);
  TPO_CK_LAUNCH();
  kb_unpack<<<b->nctas[BK_UNPACK], 256, 0, st>>>(jobs_of(b, BK_UNPACK), b->njobs[BK_UNPACK],
                                                  b->d_designs);
  TPO_CK_LAUNCH();
  kb_sens<<<b->nctas[BK_SENS], S_THREADS, 0, st>>>(jobs_of(b, BK_SENS), b->njobs[BK_SENS],
                                                     b->d_designs);
  TPO_CK_LAUNCH();
  kb_filter<<<b->nctas[BK_FILTER], F_THREADS, b->filter_smem, st>>>(
      jobs_of(b, BK_FILTER), b->njobs[BK_FILTER], b->d_designs, 1);
  TPO_CK_LAUNCH();
  kb_oc<<<b->n_slots, OCB_THREADS, 0, st>>>(b->d_designs, b->n_slots);
  TPO_CK_LAUNCH();
  kb_finish<<<cdiv(b->n_slots, 128), 128, 0, st>>>(b->d_designs, b->n_slots, b->d_status,
                                                   b->d_flag + 2);
  TPO_CK_LAUNCH();
  return TPO_OK;
}

int batch_body_any(tpo_batch *b, cudaStream_t st, cudaGraphConditionalHandle h, int use_h,
                   bool cond = true, int steps = kBatchSteps) {
  switch (b->cfg.precond) {
    case TPO_PRECOND_NONE: return batch_body<TPO_PRECOND_NONE>(b, st, h, use_h, cond, steps);
    case TPO_PRECOND_JACOBI: return batch_body<TPO_PRECOND_JACOBI>(b, st, h, use_h, cond, steps);
    default: return batch_body<TPO_PRECOND_NODAL_BLOCK>(b, st, h, use_h, cond, steps);
  }
}

// one round of continuous batching: PRE designs start their OC iteration,
// every SOLVE design advances one loop body, designs whose solve stopped
// finish their OC iteration
int batch_round_launches(tpo_batch *b, cudaStream_t st) {
  int rc = batch_prefix(b, st);
  if (!rc) rc = batch_body_any(b, st, 0, 0, false, b->round_steps);
  if (!rc) rc = batch_suffix(b, st);
  return rc;
}

// PCG loop driven from the host: bodies are enqueued two ahead of the flag reads
int batch_pcg_host(tpo_batch *b, cudaStream_t st) {
  bool pending[2] = {false, false};
  auto issue = [&](int slot) -> int {
    int rc = batch_body_any(b, st, 0, 0);
    if (rc) return rc;
    TPO_CK(cudaMemcpyAsync(b->h_flag + 4 * slot, b->d_flag, 2 * sizeof(int),
                           cudaMemcpyDeviceToHost, st));
    TPO_CK(cudaEventRecord(b->ev[slot], st));
    pending[slot] = true;
    return TPO_OK;
  };
  int rc;
  if ((rc = issue(0)) || (rc = issue(1))) return rc;
  int cur = 0;
  while (pending[cur]) {
    TPO_CK(cudaEventSynchronize(b->ev[cur]));
    pending[cur] = false;
    if (b->h_flag[4 * cur] == 0) break;
    if ((rc = issue(cur))) return rc;
    cur ^= 1;
  }
  TPO_CK(cudaStreamSynchronize(st));
  return TPO_OK;
}

// one CUDA graph per OC iteration: prefix, a while node over the PCG body, suffix
int batch_build_graph(tpo_batch *b) {
  cudaGraph_t g;
  TPO_CK(cudaGraphCreate(&g, 0));
  b->graph = g;
  cudaGraphConditionalHandle h;
  TPO_CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaStream_t cs = b->cap;
  TPO_CK(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = batch_prefix(b, cs);
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaStreamCaptureStatus cst;
  cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &ndeps);
  std::vector<cudaGraphNode_t> pre(deps, deps + (e == cudaSuccess ? ndeps : 0));
  cudaGraph_t tmp;
  TPO_CK(cudaStreamEndCapture(cs, &tmp));
  if (rc) return rc;
  TPO_CK(e);
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  TPO_CK(cudaGraphAddNode(&cnode, g, pre.data(), pre.size(), &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  TPO_CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed));
  rc = batch_body_any(b, cs, h, 1);
  TPO_CK(cudaStreamEndCapture(cs, &tmp));
  if (rc) return rc;
  TPO_CK(cudaStreamBeginCaptureToGraph(cs, g, &cnode, nullptr, 1, cudaStreamCaptureModeRelaxed));
  rc = batch_suffix(b, cs);
  TPO_CK(cudaStreamEndCapture(cs, &tmp));
  if (rc) return rc;
  TPO_CK(cudaGraphInstantiate(&b->gexec, g, 0));
  return TPO_OK;
}

int batch_build_round_graph(tpo_batch *b) {
  cudaStream_t cs = b->cap;
  TPO_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
  int rc = batch_round_launches(b, cs);
  cudaGraph_t g;
  TPO_CK(cudaStreamEndCapture(cs, &g));
  if (rc) {
    cudaGraphDestroy(g);
    return rc;
  }
  cudaError_t e = cudaGraphInstantiate(&b->rexec, g, 0);
  cudaGraphDestroy(g);
  TPO_CK(e);
  return TPO_OK;
}

int batch_read_status(tpo_batch *b, cudaStream_t st) {
  TPO_CK(cudaMemcpyAsync(b->h_status.data(), b->d_status, 2 * (size_t)b->n_slots * sizeof(int),
                         cudaMemcpyDeviceToHost, st));
  TPO_CK(cudaMemcpyAsync(b->h_flag + 8, b->d_flag, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  TPO_CK(cudaStreamSynchronize(st));
  for (int s = 0; s < b->n_slots; ++s)
    if (b->used[s] && !b->h_status[2 * s + 1] && b->rec[s].active) {
      b->rec[s].active = 0;  // finished on the device: drop it from the job tables
      b->dirty = true;
    }
  if (b->h_flag[10]) return fail(TPO_ERR_TIMEOUT, "a TMA pipeline wait ran out of time");
  if (b->h_flag[9]) return fail(TPO_ERR_TIMEOUT, "batched PCG loop stopped at its body limit");
  return TPO_OK;
}

__global__ void kb_fill(double *p, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

extern "C" {

size_t tpo_batch_workspace_bytes(int32_t max_designs) {
  if (max_designs < 1) return 0;
  Carve cv(nullptr);
  cv.take<BDesign>((size_t)max_designs);
  cv.take<BJob>((size_t)kBK * max_designs);
  cv.take<int>(4);
  cv.take<unsigned>(1);
  cv.take<int>(2 * (size_t)max_designs);
  return cv.off;
}

size_t tpo_batch_design_workspace_bytes(const tpo_batch_design *d, tpo_batch_layout *layout) {
  if (check_design(d)) return 0;
  // carve over a stand-in base address (never dereferenced) to read the offsets
  char *base = reinterpret_cast<char *>(kAlign);
  const DesignLayout L = carve_design(base, d);
  if (layout) {
    layout->rho = (size_t)(reinterpret_cast<char *>(L.rho) - base);
    layout->rho_phys = (size_t)(reinterpret_cast<char *>(L.rho_phys) - base);
    layout->u = (size_t)(reinterpret_cast<char *>(L.u) - base);
    layout->hist = (size_t)(reinterpret_cast<char *>(L.hist) - base);
  }
  return L.bytes;
}

int tpo_batch_create(int32_t max_designs, const tpo_batch_cfg *cfg, void *ws, size_t ws_bytes,
                     tpo_batch **out) {
  if (!cfg || !out || !ws) return fail(TPO_ERR_ARGS, "NULL argument");
  *out = nullptr;
  if (max_designs < 1) return fail(TPO_ERR_ARGS, "max_designs must be >= 1");
  if (cfg->precision != TPO_PRECISION_MIXED)
    return fail(TPO_ERR_ARGS, "batched designs run the mixed form only");
  if (cfg->precond != TPO_PRECOND_NONE && cfg->precond != TPO_PRECOND_JACOBI &&
      cfg->precond != TPO_PRECOND_NODAL_BLOCK)
    return fail(TPO_ERR_ARGS, "batched designs take a point preconditioner");
  if (!aligned(ws, kAlign)) return fail(TPO_ERR_ARGS, "misaligned workspace");
  if (ws_bytes < tpo_batch_workspace_bytes(max_designs))
    return fail(TPO_ERR_WORKSPACE, "batch workspace too small");
  int dev;
  int rc = need_stiffness(&dev);
  if (rc) return rc;
  tpo_batch *b = new tpo_batch();
  b->dev = dev;
  b->max_designs = max_designs;
  b->cfg = *cfg;
  if (cfg->stencil_cols > 0) b->Ls = std::max(kMinLs, (int)cfg->stencil_cols);
  if (cfg->update_cols > 0) b->Lu = std::max(kMinLu, (int)cfg->update_cols);
  if (cfg->round_steps > 0) b->round_steps = std::min(1024, (int)cfg->round_steps);
  Carve cv(ws);
  b->d_designs = cv.take<BDesign>((size_t)max_designs);
  b->d_jobs = cv.take<BJob>((size_t)kBK * max_designs);
  b->d_flag = cv.take<int>(4);
  b->d_bodies = cv.take<unsigned>(1);
  b->d_status = cv.take<int>(2 * (size_t)max_designs);
  b->rec.resize(max_designs);
  b->used.assign(max_designs, 0);
  b->h_status.assign(2 * (size_t)max_designs, 0);
  auto cleanup = [&](int code) {
    tpo_batch_destroy(b);
    return code;
  };
  if (cudaHostAlloc(reinterpret_cast<void **>(&b->h_flag), 16 * sizeof(int),
                    cudaHostAllocDefault) != cudaSuccess)
    return cleanup(fail(TPO_ERR_CUDA, "pinned flag allocation failed"));
  for (int i = 0; i < 2; ++i)
    if (cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming) != cudaSuccess)
      return cleanup(fail(TPO_ERR_CUDA, "event creation failed"));
  if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(TPO_ERR_CUDA, "stream creation failed"));
  if (cudaMemset(ws, 0, tpo_batch_workspace_bytes(max_designs)) != cudaSuccess)
    return cleanup(fail(TPO_ERR_CUDA, "workspace clear failed"));
  switch (cfg->precond) {
    case TPO_PRECOND_NONE: rc = batch_set_attrs<TPO_PRECOND_NONE>(); break;
    case TPO_PRECOND_JACOBI: rc = batch_set_attrs<TPO_PRECOND_JACOBI>(); break;
    default: rc = batch_set_attrs<TPO_PRECOND_NODAL_BLOCK>(); break;
  }
  if (rc) return cleanup(rc);
  *out = b;
  return TPO_OK;
}

int tpo_batch_destroy(tpo_batch *b) {
  if (!b) return TPO_OK;
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->rexec) cudaGraphExecDestroy(b->rexec);
  for (int i = 0; i < 2; ++i)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->h_flag) cudaFreeHost(b->h_flag);
  delete b;
  return TPO_OK;
}

int tpo_batch_add(tpo_batch *b, const tpo_batch_design *d, const double *f, const uint8_t *fixed,
                  void *dws, size_t dws_bytes, tpo_stream s, int32_t *slot_out) {
  if (!b || !f || !fixed || !dws || !slot_out) return fail(TPO_ERR_ARGS, "NULL argument");
  int rc = check_design(d);
  if (rc) return rc;
  if (!aligned(dws, kAlign) || !aligned(f, 16)) return fail(TPO_ERR_ARGS, "misaligned pointer");
  const DesignLayout L = carve_design(dws, d);
  if (dws_bytes < L.bytes) return fail(TPO_ERR_WORKSPACE, "design workspace too small");
  int slot = -1;
  for (int i = 0; i < b->max_designs; ++i)
    if (!b->used[i]) {
      slot = i;
      break;
    }
  if (slot < 0) return fail(TPO_ERR_ARGS, "batch is full (%d designs)", b->max_designs);
  cudaStream_t st = static_cast<cudaStream_t>(s);
  const int nx = d->nelx, ny = d->nely, P = pad_pitch(ny);
  const size_t NN = (size_t)(nx + 1) * P, E = (size_t)nx * ny;
  // resident state: zero everything, then density, mask and load
  TPO_CK(cudaMemsetAsync(dws, 0, L.bytes, st));
  kb_fill<<<flat_grid(E, 256, sm_count() * 8), 256, 0, st>>>(L.rho, E, d->rho0);
  TPO_CK_LAUNCH();
  const dim3 fg = flat_grid(NN, 256, sm_count() * 16);
  k_pack_mask<<<fg, 256, 0, st>>>(nx, ny, P, fixed, L.mask);
  TPO_CK_LAUNCH();
  k_pack_nodes<double><<<fg, 256, 0, st>>>(nx, ny, P, f, L.fp);
  TPO_CK_LAUNCH();
  BDesign D{};
  D.nx = nx;
  D.ny = ny;
  D.P = P;
  D.active = 1;
  D.it = 0;
  D.max_it = d->max_oc_iter;
  D.R = (int)std::ceil(d->rmin);
  D.max_cg = d->max_cg_iter;
  D.max_outer = d->max_outer;
  D.e_min = d->e_min;
  D.pen = d->penalty;
  D.volfrac = d->volfrac;
  D.move = d->move;
  D.rmin = d->rmin;
  D.tol = d->tol;
  D.tol_sq = d->cg_tol * d->cg_tol * d->f_norm_sq;
  D.rupd2 = d->inner_tol * d->inner_tol;
  D.rho = L.rho;
  D.rho_phys = L.rho_phys;
  D.dc = L.dc;
  D.dc_filt = L.dc_filt;
  D.u = L.u;
  D.hist = L.hist;
  D.mask = L.mask;
  D.up = L.up;
  D.fp = L.fp;
  D.s64 = L.s64;
  D.s32 = L.s32;
  D.fr = L.fr;
  D.fpa = L.fpa;
  D.fpb = L.fpb;
  D.fap = L.fap;
  D.fz = L.fz;
  D.ctl = L.ctl;
  D.octl = L.octl;
  D.part = L.part;
  D.phase = PH_PRE;
  D.sc = L.sc;
  D.spart = L.spart;
  D.scal = L.scal;
  b->rec[slot] = D;
  TPO_CK(cudaMemcpyAsync(b->d_designs + slot, &b->rec[slot], sizeof(BDesign),
                         cudaMemcpyHostToDevice, st));
  const int stat[2] = {0, 1};
  TPO_CK(cudaMemcpyAsync(b->d_status + 2 * slot, stat, sizeof(stat), cudaMemcpyHostToDevice, st));
  TPO_CK(cudaStreamSynchronize(st));
  b->used[slot] = 1;
  b->h_status[2 * slot] = 0;
  b->h_status[2 * slot + 1] = 1;
  b->n_slots = std::max(b->n_slots, slot + 1);
  b->dirty = true;
  *slot_out = slot;
  return TPO_OK;
}

int tpo_batch_remove(tpo_batch *b, int32_t slot) {
  if (!b || slot < 0 || slot >= b->max_designs || !b->used[slot])
    return fail(TPO_ERR_ARGS, "no design in slot %d", slot);
  const int zero = 0;
  TPO_CK(cudaMemcpy(&b->d_designs[slot].active, &zero, sizeof(int), cudaMemcpyHostToDevice));
  b->used[slot] = 0;
  b->rec[slot].active = 0;
  b->h_status[2 * slot + 1] = 0;
  while (b->n_slots > 0 && !b->used[b->n_slots - 1]) --b->n_slots;
  b->dirty = true;
  return TPO_OK;
}

int tpo_batch_set_step_period(tpo_batch *b, int32_t slot, int32_t period) {
  if (!b || slot < 0 || slot >= b->max_designs || !b->used[slot])
    return fail(TPO_ERR_ARGS, "no design in slot %d", slot);
  if (period < 1) return fail(TPO_ERR_ARGS, "the step period must be >= 1");
  b->rec[slot].period = period;
  TPO_CK(cudaMemcpy(&b->d_designs[slot].period, &period, sizeof(int), cudaMemcpyHostToDevice));
  return TPO_OK;
}

int tpo_batch_set_tiles(tpo_batch *b, int32_t stencil_cols, int32_t update_cols) {
  if (!b || stencil_cols < kMinLs || update_cols < kMinLu)
    return fail(TPO_ERR_ARGS, "strip lengths must be >= %d (stencil) and >= %d (update)", kMinLs,
                kMinLu);
  b->Ls = stencil_cols;
  b->Lu = update_cols;
  b->dirty = true;
  return TPO_OK;
}

int tpo_batch_oc_iteration(tpo_batch *b, tpo_stream s) {
  if (!b) return fail(TPO_ERR_ARGS, "batch is NULL");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  int rc;
  if (b->dirty && (rc = batch_rebuild(b, st))) return rc;
  if (b->nctas[BK_FILTER] == 0) return TPO_OK;  // nothing active
  if (b->cfg.use_graph) {
    if (!b->gexec && (rc = batch_build_graph(b))) return rc;
    TPO_CK(cudaGraphLaunch(b->gexec, st));
  } else {
    if ((rc = batch_prefix(b, st))) return rc;
    if ((rc = batch_pcg_host(b, st))) return rc;
    if ((rc = batch_suffix(b, st))) return rc;
  }
  return batch_read_status(b, st);
}

int tpo_batch_round(tpo_batch *b, int32_t rounds, tpo_stream s) {
  if (!b || rounds < 1) return fail(TPO_ERR_ARGS, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  int rc;
  if (b->dirty && (rc = batch_rebuild(b, st))) return rc;
  if (b->nctas[BK_FILTER] == 0) return TPO_OK;
  for (int i = 0; i < rounds; ++i) {
    if (b->cfg.use_graph) {
      if (!b->rexec && (rc = batch_build_round_graph(b))) return rc;
      TPO_CK(cudaGraphLaunch(b->rexec, st));
    } else if ((rc = batch_round_launches(b, st))) {
      return rc;
    }
  }
  return batch_read_status(b, st);
}

int tpo_batch_states(tpo_batch *b, int32_t n, int32_t *it_out, int32_t *active_out) {
  if (!b || n < 0 || n > b->max_designs) return fail(TPO_ERR_ARGS, "bad arguments");
  for (int i = 0; i < n; ++i) {
    const bool u = b->used[i];
    if (it_out) it_out[i] = u ? b->h_status[2 * i] : -1;
    if (active_out) active_out[i] = u ? b->h_status[2 * i + 1] : 0;
  }
  return TPO_OK;
}

// Times `steps` PCG steps (direction + update, every active design) with the
// current tiles. It advances the designs' PCG state: call it on a scratch
// batch (the autotuner builds one), not on a batch whose results are wanted.
int tpo_batch_time_steps(tpo_batch *b, int32_t steps, tpo_stream s, float *ms_out) {
  if (!b || steps < 1 || !ms_out) return fail(TPO_ERR_ARGS, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(s);
  int rc;
  if (b->dirty && (rc = batch_rebuild(b, st))) return rc;
  if (b->nctas[BK_FILTER] == 0) return fail(TPO_ERR_ARGS, "no active design");
  if ((rc = batch_prefix(b, st))) return rc;
  if ((rc = batch_body_any(b, st, 0, 0))) return rc;  // FP64 residual, first steps
  // the events are released on every path out of the timed region
  struct Events {
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  TPO_CK(cudaEventCreate(&ev.e[0]));
  TPO_CK(cudaEventCreate(&ev.e[1]));
  TPO_CK(cudaEventRecord(ev.e[0], st));
  for (int i = 0; i < steps; i += kBatchSteps)
    if ((rc = batch_body_any(b, st, 0, 0))) return rc;
  TPO_CK(cudaEventRecord(ev.e[1], st));
  TPO_CK(cudaEventSynchronize(ev.e[1]));
  float ms = 0.f;
  TPO_CK(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
  *ms_out = ms;
  return TPO_OK;
}

}  // extern "C"
