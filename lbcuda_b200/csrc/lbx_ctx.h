// lbx_ctx.h — the context behind the opaque `void* ctx` of include/lbx.h.
//
// The reference keeps its state as module-global device arrays
// (kernels_fluid.CUF:9-48) with a 1-cell halo, two ping-pong copies of the
// populations indexed by `flip`, FP32 densities and int8 flags.  Here the
// state lives in one context per simulation:
//   pops[2]   two SoA population buffers, [component][direction][z][y][x],
//             no halo (periodic wrap is index arithmetic), storage type S.
//             Buffer `cur` holds the post-collision populations of the last
//             step (pull convention: the next step gathers f_l(x - e_l)).
//   phi       phase field (rhoR - rhoB)/(rhoR + rhoB) of the current step
//             (only the two-pass colour-gradient path and the particle path).
//   rho[2]    FP32/FP64 densities (particle path, readback).
//   flags[2]  int8 cell flags of the current and previous step.
//   split[2]  (sum / predicted-split storage) per cell, the phase field that
//             the pairs of pops[i] pulled by that cell were encoded against.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

#include "../../include/lbx.h"

namespace lbx {

struct ParticleState;  // lbx_particles.cu

struct Ctx {
  lbx_params p;
  int nx = 0, ny = 0, nz = 0;
  int64_t n = 0;            // interior cells
  int ncomp = 1;            // 1 (BGK) or 2 (CG)
  int q = 19;               // populations per component: 19, or 27 for the D3Q27 models
  int storage = LBX_STORE_F32;
  bool sd = false;  // LBX_STORE_F16_SD / LBX_STORE_BF16_SD: sum / difference pairs
  bool sdp = false;  // LBX_STORE_F16_SDP / _BF16_SDP: sum / predicted-split pairs (sd is set too)
  float* split[2] = {nullptr, nullptr};  // sdp: phase field each cell decodes the pairs of pops[i] it pulls with
  size_t elem = 4;          // bytes per stored population
  void* pops[2] = {nullptr, nullptr};
  int cur = 0;              // buffer holding the current state
  void* phi = nullptr;      // float or double, n
  void* rho[2] = {nullptr, nullptr};
  int8_t* flags[2] = {nullptr, nullptr};
  int fcur = 0;             // flags slot of the current step
  unsigned long long* d_err = nullptr;
  cudaStream_t stream = nullptr;
  int64_t step = 0;
  int fused = 2;            // colour-gradient schedule: 0 two passes, 1 first single-pass kernel, 2 lean single pass
  int lean_shape = 0;       // lean kernel CTA: 0 = 32x8 (2 per SM), 1 = 32x16
  int lean_zlen = 0;        // z-segment length of the lean kernel (0 = automatic)
  int lean_copies = 1;      // 16-bit pulls: 1 = 16-byte box granules (when nx % 4 == 0), 0 = one copy per pull
  // z-slab of a decomposed box: the step computes planes [zlo, zhi) only (the
  // others are halo planes written by the exchange); zhi == 0: every plane
  int zlo = 0, zhi = 0;
  void* lean_plan = nullptr;  // device table of the lean kernel's paired segments (int4 per CTA), or null
  int lean_plan_n = 0;
  int64_t lean_plan_key = 0;
  // timing of the dominant kernel (opt-in)
  int kt_on = 0;
  std::vector<cudaEvent_t> kt_ev;
  int kt_n = 0;
  double kt_ms = 0.0;
  int64_t kt_launches = 0;
  ParticleState* part = nullptr;
  // staging buffer of the host-buffer entry points (lbx_set_fields,
  // lbx_get_fields, ...), kept between calls and grown on demand
  void* io = nullptr;
  size_t io_bytes = 0;
};

// lbx_fluid.cu
int fluid_alloc(Ctx& c);
void fluid_free(Ctx& c);
int fluid_set_fields(Ctx& c, const float* d_rhoR, const float* d_rhoB, float vx, float vy, float vz);
int fluid_set_pops(Ctx& c, const float* d_pR, const float* d_pB);
int fluid_init_rho(Ctx& c);
int fluid_collide_stream(Ctx& c);
int fluid_bgk(Ctx& c);
int fluid_step(Ctx& c);
int fluid_get_fields(Ctx& c, void* d_rR, void* d_rB, void* d_vel, void* d_phase, int f64);
int fluid_get_pops(Ctx& c, float* d_pR, float* d_pB);
int fluid_get_sums(Ctx& c, double* d_out5);
int fluid_lean(Ctx& c);
int fluid_lean_particles(Ctx& c, int fo, int fn);
void kt_begin(Ctx& c);
void kt_end(Ctx& c);

}  // namespace lbx
