// lbx_ensemble.cu — many independent boxes of uneven size advanced together
// (no counterpart in the reference, which runs one compile-time cubic box).
//
// Every box is a full context (include/lbx.h), so its fields, spheres and
// closure are set and read with the ordinary entry points.  A step of the
// ensemble forks from the ensemble stream to the stream of every box with
// spheres, runs that box's sphere pre-kernels there, joins, launches ONE
// persistent colour-gradient kernel for the fluid of all boxes
// (k_cg_lean_multi: CTAs take (box, column, z-segment) work items, longest
// first) on the ensemble stream, then forks and joins again around the sphere
// post-kernels.  The boxes' small sphere kernels thus run side by side
// instead of one after the other.  Two consecutive steps (the ping-pong
// parity) are captured once into a CUDA graph (the forks become parallel
// branches) and replayed, so the host issues one graph launch per two steps.  lbx_ensemble_tune times the
// fused fluid kernel of each candidate CTA shape and z-segment length on the
// boxes themselves and keeps the fastest.
#include <algorithm>
#include <new>
#include <vector>

#include "lbx_device.cuh"

namespace lbx {

template <typename C> struct LeanConst;
template <typename C> struct LeanPart;
template <typename C> struct BoxDesc;
struct WorkItem;
template <typename C> LeanConst<C> make_lean(const Ctx& c);

int particles_active(const Ctx& c);
int particles_pre(Ctx& c, bool forks);
int particles_post(Ctx& c, bool forks);

// implemented in lbx_fused.cu
int ensemble_launch(const std::vector<Ctx*>& boxes, int shape, const std::vector<int>& zlen, void* d_desc,
                    void* d_work, int nwork, cudaStream_t stream, int build_only, int parity);

}  // namespace lbx

namespace {

struct Ensemble {
  std::vector<lbx::Ctx*> boxes;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;       // ensemble stream -> box streams
  std::vector<cudaEvent_t> join;    // box stream -> ensemble stream
  int shape = 0;                 // 0: 32x8 CTAs, 1: 32x16
  std::vector<int> zlen;         // per box
  void* d_desc[2] = {nullptr, nullptr};
  void* d_work[2] = {nullptr, nullptr};
  int nwork = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool tables_ok = false;
};

void drop_graph(Ensemble& e) {
  if (e.exec) cudaGraphExecDestroy(e.exec);
  if (e.graph) cudaGraphDestroy(e.graph);
  e.exec = nullptr;
  e.graph = nullptr;
}

int build_tables(Ensemble& e) {
  for (int p = 0; p < 2; ++p) {
    int rc = lbx::ensemble_launch(e.boxes, e.shape, e.zlen, e.d_desc[p], e.d_work[p], 0, e.stream, 1, p);
    if (rc < 0) return rc;
    e.nwork = rc;
  }
  e.tables_ok = true;
  return 0;
}

// run `part` (a sphere stage) of every box with spheres on the box's own
// stream, between a fork from and a join into the ensemble stream
template <typename F>
int boxes_side_by_side(Ensemble& e, F&& part) {
  if (cudaEventRecord(e.fork, e.stream) != cudaSuccess) return LBX_ERR_CUDA;
  for (size_t b = 0; b < e.boxes.size(); ++b) {
    lbx::Ctx* c = e.boxes[b];
    if (!lbx::particles_active(*c)) continue;
    if (cudaStreamWaitEvent(c->stream, e.fork, 0) != cudaSuccess) return LBX_ERR_CUDA;
    int rc = part(*c);
    if (rc) return rc;
    if (cudaEventRecord(e.join[b], c->stream) != cudaSuccess ||
        cudaStreamWaitEvent(e.stream, e.join[b], 0) != cudaSuccess)
      return LBX_ERR_CUDA;
  }
  return 0;
}

// one step of every box (eager, or recorded while the ensemble stream is
// being captured)
// ta / tb (optional): events recorded on the ensemble stream around the
// fused fluid launch, the only part of a step the tuner's choice changes
int step_once(Ensemble& e, cudaEvent_t ta = nullptr, cudaEvent_t tb = nullptr) {
  if (!e.tables_ok) {
    int rc = build_tables(e);
    if (rc) return rc;
  }
  const int parity = e.boxes[0]->cur;
  for (auto* c : e.boxes)
    if (c->cur != parity) return LBX_ERR_STATE;  // boxes must be stepped together
  // each box's sphere stages on its own stream only (no second stream per box)
  int rc = boxes_side_by_side(e, [](lbx::Ctx& c) { return lbx::particles_pre(c, false); });
  if (rc) return rc;
  if (ta) cudaEventRecord(ta, e.stream);
  rc = lbx::ensemble_launch(e.boxes, e.shape, e.zlen, e.d_desc[parity], e.d_work[parity], e.nwork, e.stream, 0,
                            parity);
  if (tb) cudaEventRecord(tb, e.stream);
  if (rc) return rc;
  rc = boxes_side_by_side(e, [](lbx::Ctx& c) { return lbx::particles_post(c, false); });
  if (rc) return rc;
  for (auto* c : e.boxes)
    if (!lbx::particles_active(*c)) {
      c->cur = 1 - c->cur;
      c->step += 1;
    }
  return 0;
}

// host-side join: work the caller queued on a box (set / get calls) is done
// before the ensemble stream (or a capture of it) starts a step
int settle_boxes(Ensemble& e) {
  for (auto* c : e.boxes)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return LBX_ERR_CUDA;
  return 0;
}

}  // namespace

extern "C" {

int lbx_ensemble_create(int32_t nbox, const lbx_params* params, void** out) {
  if (!params || !out || nbox < 1) return LBX_ERR_ARG;
  *out = nullptr;
  for (int i = 1; i < nbox; ++i)
    if (params[i].storage != params[0].storage || params[i].model != LBX_MODEL_CG ||
        params[i].tauR != params[0].tauR || params[i].tauB != params[0].tauB || params[i].sigma != params[0].sigma ||
        params[i].beta != params[0].beta || params[i].rho0R != params[0].rho0R || params[i].rho0B != params[0].rho0B)
      return LBX_ERR_ARG;  // one fluid kernel (and its constants) for every box
  if (params[0].model != LBX_MODEL_CG) return LBX_ERR_ARG;
  // sum / predicted-split pairs: single boxes without spheres only
  if (params[0].storage == LBX_STORE_F16_SDP || params[0].storage == LBX_STORE_BF16_SDP) return LBX_ERR_ARG;
  Ensemble* e = new (std::nothrow) Ensemble();
  if (!e) return LBX_ERR_ALLOC;
  int rc = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess ? 0 : LBX_ERR_CUDA;
  if (!rc && cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) rc = LBX_ERR_CUDA;
  for (int i = 0; i < nbox && !rc; ++i) {
    void* h = nullptr;
    rc = lbx_create(&params[i], &h);
    if (rc) break;
    auto* c = static_cast<lbx::Ctx*>(h);
    c->fused = 2;  // each box keeps its own stream for its sphere kernels
    e->boxes.push_back(c);
    e->zlen.push_back(std::min(c->nz, 16));
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) rc = LBX_ERR_CUDA;
    e->join.push_back(ev);
  }
  size_t desc_bytes = 512 * size_t(nbox), work_cap = 0;
  for (auto* c : e->boxes) work_cap += size_t((c->nx + 31) / 32) * ((c->ny + 7) / 8) * c->nz;
  for (int p = 0; p < 2 && !rc; ++p) {
    if (cudaMalloc(&e->d_desc[p], desc_bytes) != cudaSuccess) rc = LBX_ERR_ALLOC;
    if (!rc && cudaMalloc(&e->d_work[p], work_cap * 20 + 64) != cudaSuccess) rc = LBX_ERR_ALLOC;
  }
  if (rc) {
    *out = e;
    lbx_ensemble_destroy(e);
    *out = nullptr;
    return rc;
  }
  *out = e;
  return 0;
}

int lbx_ensemble_destroy(void* ens) {
  Ensemble* e = static_cast<Ensemble*>(ens);
  if (!e) return LBX_ERR_ARG;
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graph(*e);
  for (auto* c : e->boxes) lbx_destroy(c);
  for (auto ev : e->join)
    if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  for (int p = 0; p < 2; ++p) {
    if (e->d_desc[p]) cudaFree(e->d_desc[p]);
    if (e->d_work[p]) cudaFree(e->d_work[p]);
  }
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return 0;
}

int lbx_ensemble_box(void* ens, int32_t i, void** ctx) {
  Ensemble* e = static_cast<Ensemble*>(ens);
  if (!e || !ctx || i < 0 || i >= int(e->boxes.size())) return LBX_ERR_ARG;
  *ctx = e->boxes[size_t(i)];
  drop_graph(*e);  // the caller may change the boxes' state
  return 0;
}

int lbx_ensemble_step(void* ens, int32_t nsteps) {
  Ensemble* e = static_cast<Ensemble*>(ens);
  if (!e || nsteps < 0) return LBX_ERR_ARG;
  int rc = settle_boxes(*e);
  if (rc) return rc;
  int done = 0;
  if (nsteps >= 2 && e->boxes[0]->cur == 0) {
    if (!e->exec) {
      if (!e->tables_ok && (rc = build_tables(*e))) return rc;
      // capture two steps: the buffers come back to the same parity
      if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return LBX_ERR_CUDA;
      int r1 = step_once(*e);
      int r2 = r1 ? r1 : step_once(*e);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
      // the captured launches did not run: undo the host-side step bookkeeping
      for (auto* c : e->boxes) c->step -= 2;
      if (r2 || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return r2 ? r2 : LBX_ERR_CUDA;
      }
      e->graph = g;
      if (cudaGraphInstantiate(&e->exec, e->graph, 0) != cudaSuccess) {
        drop_graph(*e);
        return LBX_ERR_CUDA;
      }
    }
    for (; done + 2 <= nsteps; done += 2) {
      if (cudaGraphLaunch(e->exec, e->stream) != cudaSuccess) return LBX_ERR_CUDA;
      for (auto* c : e->boxes) c->step += 2;
    }
  }
  for (; done < nsteps; ++done)
    if ((rc = step_once(*e))) return rc;
  // later calls on a box (on its own stream) come after these steps
  if (cudaEventRecord(e->fork, e->stream) != cudaSuccess) return LBX_ERR_CUDA;
  for (auto* c : e->boxes)
    if (cudaStreamWaitEvent(c->stream, e->fork, 0) != cudaSuccess) return LBX_ERR_CUDA;
  return 0;
}

// Time steps of the ensemble on its stream (CUDA events).
int lbx_ensemble_time(void* ens, int32_t nsteps, double* ms) {
  Ensemble* e = static_cast<Ensemble*>(ens);
  if (!e || nsteps < 0) return LBX_ERR_ARG;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, e->stream);
  int rc = lbx_ensemble_step(ens, nsteps);
  cudaEventRecord(b, e->stream);
  if (!rc && cudaEventSynchronize(b) != cudaSuccess) rc = LBX_ERR_CUDA;
  float t = 0.f;
  if (!rc) cudaEventElapsedTime(&t, a, b);
  if (ms) *ms = t;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

// Autotuner: for every candidate (CTA shape, z-segment length), build the
// work tables, run `trial` eager steps (always an even number, so the state
// parity is kept) and keep the fastest.  Returns the choice in chosen[2] =
// {shape, zlen} (zlen capped per box at its nz).
int lbx_ensemble_tune(void* ens, int32_t trial, int32_t* chosen, double* best_ms) {
  Ensemble* e = static_cast<Ensemble*>(ens);
  if (!e || trial < 2) return LBX_ERR_ARG;
  trial += trial & 1;
  drop_graph(*e);
  int rs = settle_boxes(*e);
  if (rs) return rs;
  const int shapes[2] = {0, 1};
  const int zl[6] = {4, 8, 16, 32, 64, 128};
  double best = 1e30;
  int bs = 0, bz = 16;
  for (int si = 0; si < 2; ++si)
    for (int zi = 0; zi < 6; ++zi) {
      e->shape = shapes[si];
      for (size_t i = 0; i < e->boxes.size(); ++i) e->zlen[i] = std::min(e->boxes[i]->nz, zl[zi]);
      e->tables_ok = false;
      int rc = build_tables(*e);
      if (rc) return rc;
      for (int w = 0; w < 2; ++w)
        if ((rc = step_once(*e))) return rc;
      // fused-kernel time only: the sphere kernels around it do not depend
      // on the candidate, and their eager launch overhead would swamp the
      // differences between candidates
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      float t = 0.f;
      for (int s = 0; s < trial && !rc; ++s) {
        rc = step_once(*e, a, b);
        if (rc) break;
        if (cudaEventSynchronize(b) != cudaSuccess) rc = LBX_ERR_CUDA;
        float ts = 0.f;
        if (!rc && cudaEventElapsedTime(&ts, a, b) != cudaSuccess) rc = LBX_ERR_CUDA;
        t += ts;
      }
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      if (rc) return rc;
      if (t < best) {
        best = t;
        bs = shapes[si];
        bz = zl[zi];
      }
    }
  e->shape = bs;
  for (size_t i = 0; i < e->boxes.size(); ++i) e->zlen[i] = std::min(e->boxes[i]->nz, bz);
  e->tables_ok = false;
  int rc = build_tables(*e);
  if (!rc) rc = settle_boxes(*e);
  if (!rc && cudaStreamSynchronize(e->stream) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (chosen) {
    chosen[0] = bs;
    chosen[1] = bz;
  }
  if (best_ms) *best_ms = best / trial;
  return rc;
}

}  // extern "C"
