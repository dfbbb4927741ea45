// lbx_api.cu — the extern "C" boundary declared in include/lbx.h.
//
// Replaces the host side of the reference's hot path: allocation and constant
// upload (setupGPUgridAndAlloc / SetConstants, main.CUF:2133-2407,
// 1043-1162), initial conditions (setupRho_Pops, main.CUF:2531-2608), the
// per-step launch sequence (main.CUF:125-308), the stop_d error protocol
// (abortOnLastErrorAndSync, main.CUF:2410-2442) and the readback used by
// OutputVTK (main.CUF:1812-1929).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>

#include "../../include/lbx.h"
#include "lbx_ctx.h"
#include "lbx_common.cuh"

namespace lbx {
int particles_create(Ctx& c);
void particles_destroy(Ctx& c);
int particles_set(Ctx& c, int n, const double* x, const double* v, const double* om, const double* q);
int particles_get(Ctx& c, double* x, double* v, double* om, double* q, double* f, double* t);
int particles_step(Ctx& c);
int particles_fluid(Ctx& c);
int part_lists(Ctx& c);
int part_flags(Ctx& c);
int part_drain(Ctx& c);
int part_rho(Ctx& c);
int part_fill(Ctx& c);
int part_virtual(Ctx& c);
int part_bb(Ctx& c, int mode);
int part_pairs(Ctx& c);
int part_integrate(Ctx& c);
int particles_set_closure(Ctx& c, const float* w);
int particles_flags_slot(const Ctx& c);
int particles_links(Ctx& c, int32_t* cell, int8_t* dir, int32_t* sph, int64_t cap, int64_t* n);
int particles_active(const Ctx& c);
}  // namespace lbx

using lbx::Ctx;

namespace {

int cuda_rc(cudaError_t e) { return e == cudaSuccess ? 0 : LBX_ERR_CUDA; }

// device error word -> status; clears it
int poll_error(Ctx& c, int32_t* code, int32_t* step, int64_t* where) {
  unsigned long long v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, c.d_err, sizeof(v), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return LBX_ERR_CUDA;
  int cd = int(v >> 56);
  if (code) *code = cd;
  if (step) *step = int32_t((v >> 32) & 0xffffff);
  if (where) *where = int64_t(v & 0xffffffffull);
  if (v) cudaMemsetAsync(c.d_err, 0, sizeof(v), c.stream);
  return 0;
}

// synchronise and fold a pending device error into the return status
int sync_status(Ctx& c) {
  cudaError_t e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return LBX_ERR_CUDA;
  unsigned long long v = 0;
  e = cudaMemcpy(&v, c.d_err, sizeof(v), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return LBX_ERR_CUDA;
  return v ? int(v >> 56) : 0;
}

// temporary device buffer for host<->device staging of one call
// Device staging area of the context for host-buffer transfers: allocated
// on first use and grown when a larger transfer comes, never per call (a
// cudaMalloc / cudaFree pair per call cost milliseconds and synchronised the
// device).
struct DevBuf {
  void* p = nullptr;
  DevBuf(lbx::Ctx* c, size_t bytes) {
    if (bytes > c->io_bytes) {
      if (c->io) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->io);
      }
      c->io = nullptr;
      c->io_bytes = 0;
      if (cudaMalloc(&c->io, bytes) != cudaSuccess) {
        c->io = nullptr;
        return;
      }
      c->io_bytes = bytes;
    }
    p = c->io;
  }
};

Ctx* as_ctx(void* ctx) { return static_cast<Ctx*>(ctx); }

}  // namespace

// Rows of `row` elements T, `rows` of them, from src (rows `sstride` apart)
// to dst (rows `dstride` apart): blockIdx.y is the row.  A 2-D memcpy between
// device buffers measured about 9 us per 2.5 MB of planes on B200, this about
// a third of that; the halo exchange runs it four times per step.
template <typename T>
__global__ void __launch_bounds__(256) k_copy_rows(const T* __restrict__ src, T* __restrict__ dst, size_t row,
                                                   size_t sstride, size_t dstride) {
  const T* s = src + size_t(blockIdx.y) * sstride;
  T* d = dst + size_t(blockIdx.y) * dstride;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < row; i += size_t(gridDim.x) * blockDim.x)
    d[i] = s[i];
}

static int copy_rows(lbx::Ctx* c, const char* src, char* dst, size_t row_bytes, size_t sstride, size_t dstride,
                     int rows) {
  const bool v16 = (row_bytes | sstride | dstride | size_t(src) | size_t(dst)) % 16 == 0;
  const size_t es = v16 ? 16 : 4;
  if ((row_bytes | sstride | dstride | size_t(src) | size_t(dst)) % es) return LBX_ERR_ARG;
  const size_t row = row_bytes / es;
  const unsigned gx = unsigned(std::min<size_t>((row + 255) / 256, 64));
  const dim3 grid(gx, unsigned(rows));
  if (v16)
    k_copy_rows<uint4><<<grid, 256, 0, c->stream>>>(reinterpret_cast<const uint4*>(src), reinterpret_cast<uint4*>(dst),
                                                    row, sstride / es, dstride / es);
  else
    k_copy_rows<unsigned><<<grid, 256, 0, c->stream>>>(reinterpret_cast<const unsigned*>(src),
                                                       reinterpret_cast<unsigned*>(dst), row, sstride / es,
                                                       dstride / es);
  return cuda_rc(cudaGetLastError());
}

extern "C" {

void lbx_default_params(lbx_params* p, int32_t nx, int32_t ny, int32_t nz) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->model = LBX_MODEL_CG;
  p->storage = LBX_STORE_F32;
  p->wetting = LBX_WET_JANUS;
  p->lrotate = 0;
  p->max_particles = 0;
  p->tau = 1.0f;
  p->tauR = 1.0f;  // dimensions_m.CUF:98-99
  p->tauB = 1.0f;
  p->sigma = 0.1f;  // dimensions_m.CUF:50
  p->beta = 0.999f;
  p->rho0R = 0.5f;
  p->rho0B = 0.5f;
  p->radius = 5.5f;             // dimensions_m.CUF:59
  p->rmass = 1.0f / 1500.0f;    // dimensions_m.CUF:60
  p->max_vel = 0.0f;
  p->hz_k = 10.0f;              // dimensions_m.CUF:77-80
  p->hz_rmin = 10.5f;
  p->hz_rcap = 9.0f;
  p->lubrication = 0;           // dimensions_m.CUF:81-84
  p->lubric_k = 10.0f;
  p->lubric_rmin = 10.0f;
  p->lubric_rcap = 9.0f;
  p->kinematic = 0;
  p->closure = 0;
  p->closure_gap_min = 0.05f;
  p->closure_gap_max = 1.5f;
  p->closure_vmax = 1.0e-3f;
  p->exact_tiles = 1;
  p->densR = 1.0f;  // noDIFFDENS values (SetConstants, main.CUF:1065-1066)
  p->densB = 1.0f;
}

int lbx_create(const lbx_params* p, void** out) {
  if (!p || !out) return LBX_ERR_ARG;
  *out = nullptr;
  if (p->nx < 3 || p->ny < 3 || p->nz < 3) return LBX_ERR_ARG;
  if (p->model < LBX_MODEL_BGK || p->model > LBX_MODEL_CG_DIFFDENS_D3Q27) return LBX_ERR_ARG;
  const bool two_dens = p->model == LBX_MODEL_CG_DIFFDENS || p->model == LBX_MODEL_CG_DIFFDENS_D3Q27;
  const bool d3q27 = p->model == LBX_MODEL_CG_D3Q27 || p->model == LBX_MODEL_CG_DIFFDENS_D3Q27;
  // the reference's sphere kernels are D3Q19 only (kernels_fluid_PART.CUF:1929-1941)
  if (d3q27 && p->max_particles > 0) return LBX_ERR_ARG;
  // SetConstants, main.CUF:1047-1061: at least one of the two densities is 1
  if (two_dens &&
      (!(p->densR > 0.0f) || !(p->densB > 0.0f) || (p->densR != 1.0f && p->densB != 1.0f)))
    return LBX_ERR_ARG;
  if (p->storage < LBX_STORE_F32 || p->storage > LBX_STORE_BF16_SDP) return LBX_ERR_ARG;
  const bool sdp = p->storage == LBX_STORE_F16_SDP || p->storage == LBX_STORE_BF16_SDP;
  const bool sd = sdp || p->storage == LBX_STORE_F16_SD || p->storage == LBX_STORE_BF16_SD;
  // sum / difference pairs: the single-pass colour-gradient kernel (with or without spheres) only;
  // sum / predicted-split pairs: without spheres
  if (sd && p->model != LBX_MODEL_CG) return LBX_ERR_ARG;
  if (sdp && p->max_particles > 0) return LBX_ERR_ARG;
  int64_t n = int64_t(p->nx) * p->ny * p->nz;
  if (n >= (int64_t(1) << 31)) return LBX_ERR_ARG;  // 32-bit cell indices
  Ctx* c = new (std::nothrow) Ctx();
  if (!c) return LBX_ERR_ALLOC;
  c->p = *p;
  c->nx = p->nx;
  c->ny = p->ny;
  c->nz = p->nz;
  c->n = n;
  c->ncomp = (p->model == LBX_MODEL_BGK) ? 1 : 2;
  c->q = d3q27 ? lbx::Q27 : lbx::Q;
  // the DIFFDENS collision and the D3Q27 lattice run on the two-pass schedule only
  if (two_dens || d3q27) c->fused = 0;
  c->storage = p->storage;
  c->sd = sd;
  c->sdp = sdp;
  if (sd) c->fused = 2;
  c->elem = (p->storage == LBX_STORE_F32) ? 4 : (p->storage == LBX_STORE_F64 ? 8 : 2);
  int rc = cuda_rc(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  if (!rc) rc = cuda_rc(cudaMalloc(&c->d_err, sizeof(unsigned long long)));
  if (!rc) rc = cuda_rc(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned long long), c->stream));
  if (!rc) rc = lbx::fluid_alloc(*c);
  if (!rc && p->max_particles > 0) rc = lbx::particles_create(*c);
  if (!rc) rc = cuda_rc(cudaStreamSynchronize(c->stream));
  if (rc) {
    lbx_destroy(c);
    return rc;
  }
  *out = c;
  return 0;
}

int lbx_destroy(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  if (c->stream) cudaStreamSynchronize(c->stream);
  lbx::particles_destroy(*c);
  lbx::fluid_free(*c);
  for (auto e : c->kt_ev) cudaEventDestroy(e);
  if (c->d_err) cudaFree(c->d_err);
  if (c->io) cudaFree(c->io);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int lbx_set_fields(void* ctx, const float* rhoR, const float* rhoB, float vx, float vy, float vz) {
  Ctx* c = as_ctx(ctx);
  if (!c || !rhoR || (c->ncomp == 2 && !rhoB)) return LBX_ERR_ARG;
  size_t bytes = size_t(c->n) * sizeof(float);
  DevBuf buf(c, bytes * c->ncomp);
  if (!buf.p) return LBX_ERR_ALLOC;
  float* dR = static_cast<float*>(buf.p);
  float* dB = (c->ncomp == 2) ? dR + c->n : nullptr;
  int rc = cuda_rc(cudaMemcpyAsync(dR, rhoR, bytes, cudaMemcpyHostToDevice, c->stream));
  if (!rc && dB) rc = cuda_rc(cudaMemcpyAsync(dB, rhoB, bytes, cudaMemcpyHostToDevice, c->stream));
  if (!rc) rc = lbx::fluid_set_fields(*c, dR, dB, vx, vy, vz);
  if (!rc) rc = cuda_rc(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned long long), c->stream));
  c->step = 0;
  if (!rc) rc = cuda_rc(cudaStreamSynchronize(c->stream));
  return rc;
}

int lbx_set_pops(void* ctx, const float* popsR, const float* popsB) {
  Ctx* c = as_ctx(ctx);
  if (!c || !popsR || (c->ncomp == 2 && !popsB)) return LBX_ERR_ARG;
  size_t bytes = size_t(c->n) * size_t(c->q) * sizeof(float);
  DevBuf buf(c, bytes * c->ncomp);
  if (!buf.p) return LBX_ERR_ALLOC;
  float* dR = static_cast<float*>(buf.p);
  float* dB = (c->ncomp == 2) ? dR + c->n * c->q : nullptr;
  int rc = cuda_rc(cudaMemcpyAsync(dR, popsR, bytes, cudaMemcpyHostToDevice, c->stream));
  if (!rc && dB) rc = cuda_rc(cudaMemcpyAsync(dB, popsB, bytes, cudaMemcpyHostToDevice, c->stream));
  if (!rc) rc = lbx::fluid_set_pops(*c, dR, dB);
  c->step = 0;
  if (!rc) rc = cuda_rc(cudaStreamSynchronize(c->stream));
  return rc;
}

int lbx_step(void* ctx, int32_t nsteps) {
  Ctx* c = as_ctx(ctx);
  if (!c || nsteps < 0) return LBX_ERR_ARG;
  const bool parts = lbx::particles_active(*c);
  for (int s = 0; s < nsteps; ++s) {
    int rc = parts ? lbx::particles_step(*c) : lbx::fluid_step(*c);
    if (rc) return rc;
  }
  return 0;
}

int lbx_init_rho(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  if (lbx::particles_active(*c)) return lbx::part_rho(*c);
  return lbx::fluid_init_rho(*c);
}

int lbx_time_step_cg(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  // with spheres the step ends in lbx_time_step_force_particles
  if (lbx::particles_active(*c)) return c->ncomp == 2 ? lbx::particles_fluid(*c) : LBX_ERR_STATE;
  int rc = lbx::fluid_collide_stream(*c);
  if (!rc) c->step += 1;
  return rc;
}

// kernel-level particle stages (main.CUF:130-240)
#define LBX_PART_STAGE(name, call)           \
  int name(void* ctx) {                      \
    Ctx* c = as_ctx(ctx);                    \
    if (!c) return LBX_ERR_ARG;              \
    if (!lbx::particles_active(*c)) return LBX_ERR_STATE; \
    return call;                             \
  }
LBX_PART_STAGE(lbx_make_list_atoms, lbx::part_lists(*c))
LBX_PART_STAGE(lbx_init_isfluid, lbx::part_flags(*c))
LBX_PART_STAGE(lbx_del_fluid, lbx::part_drain(*c))
LBX_PART_STAGE(lbx_make_fluid, lbx::part_fill(*c))
LBX_PART_STAGE(lbx_virtual_rho, lbx::part_virtual(*c))
LBX_PART_STAGE(lbx_partbb, lbx::part_bb(*c, 1))
LBX_PART_STAGE(lbx_partbb_p2n, lbx::part_bb(*c, 2))
LBX_PART_STAGE(lbx_partbb_p2n2, lbx::part_bb(*c, 4))
LBX_PART_STAGE(lbx_inter_force_particles, lbx::part_pairs(*c))
LBX_PART_STAGE(lbx_time_step_force_particles, lbx::part_integrate(*c))
#undef LBX_PART_STAGE

int lbx_time_step_bgk(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  int rc = lbx::fluid_bgk(*c);
  if (!rc) c->step += 1;
  return rc;
}

static int get_fields_impl(Ctx* c, void* rR, void* rB, void* vel, void* phase, int f64) {
  size_t es = f64 ? 8 : 4;
  size_t nb = size_t(c->n) * es;
  DevBuf buf(c, nb * 6);
  if (!buf.p) return LBX_ERR_ALLOC;
  char* d = static_cast<char*>(buf.p);
  void* dR = rR ? d : nullptr;
  void* dB = rB ? d + nb : nullptr;
  void* dV = vel ? d + 2 * nb : nullptr;
  void* dP = phase ? d + 5 * nb : nullptr;
  int rc = lbx::fluid_get_fields(*c, dR, dB, dV, dP, f64);
  if (!rc && rR) rc = cuda_rc(cudaMemcpyAsync(rR, dR, nb, cudaMemcpyDeviceToHost, c->stream));
  if (!rc && rB) rc = cuda_rc(cudaMemcpyAsync(rB, dB, nb, cudaMemcpyDeviceToHost, c->stream));
  if (!rc && vel) rc = cuda_rc(cudaMemcpyAsync(vel, dV, 3 * nb, cudaMemcpyDeviceToHost, c->stream));
  if (!rc && phase) rc = cuda_rc(cudaMemcpyAsync(phase, dP, nb, cudaMemcpyDeviceToHost, c->stream));
  if (!rc) rc = sync_status(*c);
  return rc;
}

int lbx_get_fields(void* ctx, float* rhoR, float* rhoB, float* vel, float* phase) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  return get_fields_impl(c, rhoR, rhoB, vel, phase, 0);
}

int lbx_get_fields_f64(void* ctx, double* rhoR, double* rhoB, double* vel, double* phase) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  return get_fields_impl(c, rhoR, rhoB, vel, phase, 1);
}

int lbx_get_pops(void* ctx, float* popsR, float* popsB) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  size_t nb = size_t(c->n) * size_t(c->q) * sizeof(float);
  DevBuf buf(c, nb * 2);
  if (!buf.p) return LBX_ERR_ALLOC;
  float* dR = popsR ? static_cast<float*>(buf.p) : nullptr;
  float* dB = popsB ? static_cast<float*>(buf.p) + size_t(c->n) * size_t(c->q) : nullptr;
  int rc = lbx::fluid_get_pops(*c, dR, dB);
  if (!rc && popsR) rc = cuda_rc(cudaMemcpyAsync(popsR, dR, nb, cudaMemcpyDeviceToHost, c->stream));
  if (!rc && popsB) {
    if (c->ncomp == 2) rc = cuda_rc(cudaMemcpyAsync(popsB, dB, nb, cudaMemcpyDeviceToHost, c->stream));
    else std::memset(popsB, 0, nb);
  }
  if (!rc) rc = sync_status(*c);
  return rc;
}

int lbx_get_flags(void* ctx, int8_t* flags) {
  Ctx* c = as_ctx(ctx);
  if (!c || !flags) return LBX_ERR_ARG;
  int rc = cuda_rc(cudaMemcpyAsync(flags, c->flags[lbx::particles_flags_slot(*c)], size_t(c->n),
                                   cudaMemcpyDeviceToHost, c->stream));
  if (!rc) rc = sync_status(*c);
  return rc;
}

int lbx_get_links(void* ctx, int32_t* cell, int8_t* dir, int32_t* sphere, int64_t cap, int64_t* n) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  int rc = lbx::particles_links(*c, cell, dir, sphere, cap, n);
  if (!rc) rc = sync_status(*c);
  return rc;
}

int lbx_get_sums(void* ctx, double* mass, double* momentum) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  DevBuf buf(c, 5 * sizeof(double));
  if (!buf.p) return LBX_ERR_ALLOC;
  double h[5];
  int rc = lbx::fluid_get_sums(*c, static_cast<double*>(buf.p));
  if (!rc) rc = cuda_rc(cudaMemcpyAsync(h, buf.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  if (!rc) rc = sync_status(*c);
  if (!rc) {
    if (mass) { mass[0] = h[0]; mass[1] = h[1]; }
    if (momentum) { momentum[0] = h[2]; momentum[1] = h[3]; momentum[2] = h[4]; }
  }
  return rc;
}

int lbx_set_particles(void* ctx, int32_t n, const double* xyz, const double* vel, const double* omega,
                      const double* q) {
  Ctx* c = as_ctx(ctx);
  if (!c || !xyz || n < 1) return LBX_ERR_ARG;
  if (!c->part) return LBX_ERR_STATE;
  return lbx::particles_set(*c, n, xyz, vel, omega, q);
}

int lbx_get_particles(void* ctx, double* xyz, double* vel, double* omega, double* q, double* force, double* torque) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  int rc = lbx::particles_get(*c, xyz, vel, omega, q, force, torque);
  if (!rc) rc = sync_status(*c);
  return rc;
}

int lbx_closure_set(void* ctx, const float* weights) {
  Ctx* c = as_ctx(ctx);
  if (!c || !weights) return LBX_ERR_ARG;
  return lbx::particles_set_closure(*c, weights);
}

int lbx_sync(void* ctx) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  return sync_status(*c);
}

int lbx_status(void* ctx, int32_t* code, int32_t* step, int64_t* where) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  return poll_error(*c, code, step, where);
}

int lbx_get_step(void* ctx, int64_t* step) {
  Ctx* c = as_ctx(ctx);
  if (!c || !step) return LBX_ERR_ARG;
  *step = c->step;
  return 0;
}

const char* lbx_error_string(int code) {
  switch (code) {
    case 0: return "ok";
    case LBX_ERR_CUDA: return "CUDA runtime error";
    case LBX_ERR_ARG: return "invalid argument";
    case LBX_ERR_ALLOC: return "device allocation failed";
    case LBX_ERR_STATE: return "operation not valid for this context";
    case LBX_ERR_TIMEOUT: return "device wait timed out";
    case LBX_ERR_NOSYM: return "device symbol not available";
    case LBX_DEV_RHO_RANGE: return "density out of range [-10, 10] (init_rho*_CG)";
    case LBX_DEV_BIG_FORCE: return "particle force too large (nve_lf)";
    case LBX_DEV_EXTREME_VEL: return "particle speed above MAX_PARTICLE_VEL (nve_lf)";
    case LBX_DEV_POSITION: return "particle position outside the box (nve_lf)";
    case LBX_DEV_LIST_OVERFLOW: return "too many particles near one cell block";
    case LBX_DEV_BELT_RANGE: return "belt neighbour outside the lattice";
    case LBX_DEV_WAIT_TIMEOUT: return "in-kernel wait timed out";
  }
  return "unknown error";
}

/* ---- measurement hooks used by the benchmark --------------------------- */
/* Select the colour-gradient schedule: 1 = single-pass fused kernel (default),
 * 0 = two passes (phase field, then collision). */
int lbx_set_schedule(void* ctx, int32_t fused) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  if (fused < 0 || fused > 2) return LBX_ERR_ARG;
  if (c->p.model >= LBX_MODEL_CG_DIFFDENS && fused != 0) return LBX_ERR_ARG;
  if (c->sd && fused != 2) return LBX_ERR_ARG;  // sum / difference pairs: lean kernel only
  if (c->zhi > 0 && fused != 2) return LBX_ERR_STATE;  // a z-slab steps on the lean kernel
  c->fused = fused;
  return 0;
}

/* Shape of the lean single-pass kernel: shape 0 = 32x8 cells per CTA, 1 =
 * 32x16; zlen = planes per z-segment (0 = automatic). */
int lbx_set_lean_shape(void* ctx, int32_t shape, int32_t zlen) {
  Ctx* c = as_ctx(ctx);
  if (!c || shape < 0 || shape > 1 || zlen < 0) return LBX_ERR_ARG;
  c->lean_shape = shape;
  c->lean_zlen = zlen;
  return 0;
}

/* ---- z-slab decomposition ------------------------------------------------
 * The reference splits the box into z-slabs, one MPI rank each, and swaps
 * halo planes of populations between neighbours every step
 * (main.CUF:504-1000, setupMPI.CUF:26-30).  Here a slab is a context of its
 * own planes plus two halo planes on each side; the step computes the own
 * planes only, and the host moves the halo planes between contexts or GPUs
 * (lbcuda_b200/slabs.py) through these packed copies. */
int lbx_set_zrange(void* ctx, int32_t zlo, int32_t zhi) {
  Ctx* c = as_ctx(ctx);
  if (!c) return LBX_ERR_ARG;
  if (zlo == 0 && zhi == 0) {  // the whole box again
    c->zlo = c->zhi = 0;
    return 0;
  }
  // the step pulls from planes zlo - 2 .. zhi + 1 (the phase field of the
  // planes next to the own ones): they must exist without a wrap
  if (zlo < 2 || zhi > c->nz - 2 || zlo >= zhi) return LBX_ERR_ARG;
  // the lean colour-gradient kernel only, without spheres
  if (c->ncomp != 2 || c->q != 19 || c->p.model != LBX_MODEL_CG || c->fused != 2 || lbx::particles_active(*c) ||
      c->p.max_particles > 0)
    return LBX_ERR_STATE;
  c->zlo = zlo;
  c->zhi = zhi;
  return 0;
}

static size_t pair_bytes(const Ctx& c) { return c.elem * size_t(c.ncomp); }

/* Bytes of lbx_pack_planes for nplanes planes. */
int lbx_plane_bytes(void* ctx, int32_t nplanes, int64_t* bytes) {
  Ctx* c = as_ctx(ctx);
  if (!c || !bytes || nplanes < 0) return LBX_ERR_ARG;
  const size_t cells = size_t(nplanes) * size_t(c->nx) * size_t(c->ny);
  *bytes = int64_t(cells * pair_bytes(*c) * size_t(c->q) + (c->sdp ? cells * sizeof(float) : 0));
  return 0;
}

// planes [z0, z0 + np) of the current populations <-> a packed device buffer
static int move_planes(Ctx* c, int z0, int np, char* buf, bool pack) {
  if (!c || !buf || np <= 0 || z0 < 0 || z0 + np > c->nz) return LBX_ERR_ARG;
  const size_t plane = size_t(c->nx) * size_t(c->ny), pb = pair_bytes(*c);
  const size_t width = size_t(np) * plane * pb, pitch = size_t(c->n) * pb;
  char* pops = static_cast<char*>(c->pops[c->cur]) + size_t(z0) * plane * pb;
  int rc = pack ? copy_rows(c, pops, buf, width, pitch, width, c->q) : copy_rows(c, buf, pops, width, width, pitch, c->q);
  if (!rc && c->sdp) {  // the phase field the pairs of these planes were encoded against
    char* sp = reinterpret_cast<char*>(c->split[c->cur] + size_t(z0) * plane);
    char* bs = buf + width * size_t(c->q);
    const size_t sb = size_t(np) * plane * sizeof(float);
    rc = pack ? copy_rows(c, sp, bs, sb, sb, sb, 1) : copy_rows(c, bs, sp, sb, sb, sb, 1);
  }
  return rc;
}

/* Copy planes [z0, z0 + nplanes) of the current populations (stored form,
 * all directions and components; with sum / predicted-split pairs also the
 * split field of those planes) into a packed device buffer of
 * lbx_plane_bytes bytes: direction by direction, nplanes * nx * ny pairs each.
 * Enqueued on the context's stream (lbx_sync before another stream reads it). */
int lbx_pack_planes(void* ctx, int32_t z0, int32_t nplanes, void* dev_buf) {
  return move_planes(as_ctx(ctx), z0, nplanes, static_cast<char*>(dev_buf), true);
}

/* The reverse: write a packed buffer into planes [z0, z0 + nplanes). */
int lbx_unpack_planes(void* ctx, int32_t z0, int32_t nplanes, const void* dev_buf) {
  return move_planes(as_ctx(ctx), z0, nplanes, static_cast<char*>(const_cast<void*>(dev_buf)), false);
}

/* The CUDA stream (cudaStream_t) the context enqueues all its work on, so a
 * host can order its own copies or collectives with the steps. */
int lbx_get_stream(void* ctx, void** stream) {
  Ctx* c = as_ctx(ctx);
  if (!c || !stream) return LBX_ERR_ARG;
  *stream = static_cast<void*>(c->stream);
  return 0;
}

/* Staging of the lean kernel's 16-bit pulls: 1 = box granules, 0 = one copy per pull. */
int lbx_set_lean_copies(void* ctx, int32_t mode) {
  Ctx* c = as_ctx(ctx);
  if (!c || mode < 0 || mode > 1) return LBX_ERR_ARG;
  c->lean_copies = mode;
  return 0;
}

/* Time nsteps steps on the context stream with CUDA events: total device
 * time in ms, and the summed duration of the step's dominant kernel (the
 * fused collide-stream kernel) with its launch count. */
int lbx_time_steps(void* ctx, int32_t nsteps, double* total_ms, double* kernel_ms, int64_t* kernel_launches) {
  Ctx* c = as_ctx(ctx);
  if (!c || nsteps < 0) return LBX_ERR_ARG;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  c->kt_on = kernel_ms ? 1 : 0;
  c->kt_n = 0;
  cudaEventRecord(e0, c->stream);
  int rc = lbx_step(ctx, nsteps);
  cudaEventRecord(e1, c->stream);
  if (!rc) rc = cuda_rc(cudaEventSynchronize(e1));
  float ms = 0.f;
  if (!rc) cudaEventElapsedTime(&ms, e0, e1);
  if (total_ms) *total_ms = ms;
  double kms = 0.0;
  if (!rc && c->kt_on) {
    for (int i = 0; i < c->kt_n; ++i) {
      float t = 0.f;
      cudaEventElapsedTime(&t, c->kt_ev[2 * i], c->kt_ev[2 * i + 1]);
      kms += t;
    }
  }
  if (kernel_ms) *kernel_ms = kms;
  if (kernel_launches) *kernel_launches = c->kt_n;
  c->kt_on = 0;
  c->kt_n = 0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = sync_status(*c);
  return rc;
}

}  // extern "C"
