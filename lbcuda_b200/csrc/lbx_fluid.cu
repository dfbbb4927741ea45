// lbx_fluid.cu — fluid kernels of the LBcuda hot path for sm_100a.
//
// Reference behaviour restated (paths relative to the reference project):
//   equil                         kernels_fluid_CG.CUF:30-38
//   init_rhoR_CG / init_rhoB_CG   kernels_fluid_CG.CUF:398-509
//   time_step_CG                  kernels_fluid_CG.CUF:531-848
//   flipflop*Pop0_CG, stream*_CG  kernels_fluid_CG.CUF:851-1015
//   stream_CG_x/_y/_z + fixPeriodic (halo wrap)  kernels_fluid_CG.CUF:1017-1141,
//                                 1215-1426; main.CUF:577-1000
//   time_step_BGK + stream_BGK    kernels_fluid_BGK.CUF:205-417
//   moments2Fl (readback)         write_output.f90:975-1041
//
// B200 design (not a translation): SoA populations without a halo ring,
// periodic wrap by index arithmetic, pull streaming (each thread gathers
// f_l(x - e_l) of the previous post-collision buffer, so every store is
// aligned and coalesced), one thread per cell along contiguous x rows, and
// FP16/BF16 storage of f_l - w_l*rho0 with FP32 arithmetic.
//
// The colour-gradient collision needs the phase field of all 26 neighbours at
// the same time level.  Two schedules are provided:
//   two-pass: k_cg_phi (pull + densities -> phi) then k_cg_collide;
//   single-pass: k_cg_fused, where each CTA owns a (BX x BY) column of cells
//   and marches it along z, computing the phase field of its own cells and of
//   a one-cell ring around the column from the pulled populations into a
//   rolling 3-plane shared-memory window, so phi never goes through HBM.
#include "lbx_device.cuh"

#include <cstdio>

namespace lbx {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// setupPops (kernels_fluid_CG.CUF:313-346) written in pull convention: the
// stored buffer holds, at x, the populations that streaming moves to x + e_l,
// so that the first step gathers exactly the equilibrium of the given fields
// (equilCG with two fluid densities, kernels_fluid_CG.CUF:176-178).
template <typename S, bool DD, int QQ>
__global__ void k_set_fields(S* __restrict__ A, S* __restrict__ B, Geom g, int ncomp, const float* __restrict__ rR,
                             const float* __restrict__ rB, float vx, float vy, float vz,
                             CGConst<typename Store<S>::C> K, Shift<typename Store<S>::C> sh) {
  using C = typename Store<S>::C;
  const LatticeT<C>& L = K.L;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C u = C(vx), v = C(vy), w = C(vz);
  C usq = L.half_inv_cssq * (u * u + v * v + w * w);
  if (sh.sd) {  // sum / difference pairs (single density, D3Q19)
    C f0[Q], f1[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      f0[l] = equil_u(L, C(rR[at(b, ex(l), ey(l), ez(l))]), edot(l, u, v, w), usq, l);
      f1[l] = equil_u(L, C(rB[at(b, ex(l), ey(l), ez(l))]), edot(l, u, v, w), usq, l);
    }
    rb_to_sd(f0, f1);
    if (sh.split) {  // predicted split: against the phase field of the cell that pulls the pair
#pragma unroll
      for (int l = 0; l < Q; ++l) f1[l] = f1[l] - C(sh.split[at(b, ex(l), ey(l), ez(l))]) * f0[l];
    }
    store_all(A, g, cell, 0, sh, f0);
    store_all(A, g, cell, 1, sh, f1);
#pragma unroll
    for (int l = 0; l < Q; ++l) f0[l] = f1[l] = C(0);
    store_all(B, g, cell, 0, sh, f0);
    store_all(B, g, cell, 1, sh, f1);
    return;
  }
  for (int comp = 0; comp < ncomp; ++comp) {
    const float* r = comp ? rB : rR;
#pragma unroll
    for (int l = 0; l < QQ; ++l) {
      C rho = C(r[at(b, ex(l), ey(l), ez(l))]);
      C val = DD ? equil_cg(K, rho, edot(l, u, v, w), usq, comp, l) : equil_u(L, rho, edot(l, u, v, w), usq, l);
      Store<S>::st(A + pidx(g, comp, l, cell), val, sh.at(comp, l));
      Store<S>::st(B + pidx(g, comp, l, cell), C(0), sh.at(comp, l));
    }
  }
}

// Sum / predicted-split storage: the phase field each cell decodes its pulled
// pairs with, for a state given as densities (set_fields) or as populations
// (set_pops: the phase of each cell's pulled populations).
__global__ void k_split_of_fields(Geom g, const float* __restrict__ rR, const float* __restrict__ rB, float* split) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  const float r = fmaxf(rR[i], 0.f), b = fmaxf(rB[i], 0.f);
  split[i] = (r + b > 0.f) ? (r - b) / (r + b) : 0.f;
}
template <int QQ>
__global__ void k_split_of_pops(Geom g, const float* __restrict__ pR, const float* __restrict__ pB, float* split) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  float r = 0.f, b = 0.f;
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    r += pR[size_t(l) * size_t(g.n) + size_t(i)];
    b += pB[size_t(l) * size_t(g.n) + size_t(i)];
  }
  r = fmaxf(r, 0.f);
  b = fmaxf(b, 0.f);
  split[i] = (r + b > 0.f) ? (r - b) / (r + b) : 0.f;
}

// initType 4: raw post-streaming populations, stored in pull convention
template <typename S, int QQ>
__global__ void k_set_pops(S* __restrict__ A, Geom g, int ncomp, const float* __restrict__ pR,
                           const float* __restrict__ pB, Shift<typename Store<S>::C> sh) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  if (sh.sd) {  // sum / difference pairs (D3Q19)
    C f0[Q], f1[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      f0[l] = C(pR[size_t(l) * size_t(g.n) + at(b, ex(l), ey(l), ez(l))]);
      f1[l] = C(pB[size_t(l) * size_t(g.n) + at(b, ex(l), ey(l), ez(l))]);
    }
    rb_to_sd(f0, f1);
    if (sh.split) {  // predicted split: against the phase field of the cell that pulls the pair
#pragma unroll
      for (int l = 0; l < Q; ++l) f1[l] = f1[l] - C(sh.split[at(b, ex(l), ey(l), ez(l))]) * f0[l];
    }
    store_all(A, g, cell, 0, sh, f0);
    store_all(A, g, cell, 1, sh, f1);
    return;
  }
  for (int comp = 0; comp < ncomp; ++comp) {
    const float* p = comp ? pB : pR;
#pragma unroll
    for (int l = 0; l < QQ; ++l)
      Store<S>::st(A + pidx(g, comp, l, cell), C(p[size_t(l) * size_t(g.n) + at(b, ex(l), ey(l), ez(l))]),
                   sh.at(comp, l));
  }
}

// init_rhoR_CG + init_rhoB_CG (all cells fluid) producing the phase field of
// the two-pass schedule and, optionally, the densities.
template <typename S, int QQ>
__global__ void __launch_bounds__(256) k_cg_phi(const S* __restrict__ A, Geom g, Shift<typename Store<S>::C> sh,
                                                 typename Store<S>::C* __restrict__ phi,
                                                 typename Store<S>::C* __restrict__ rhoR,
                                                 typename Store<S>::C* __restrict__ rhoB,
                                                 unsigned long long* err, int64_t step, typename Store<S>::C densR,
                                                 typename Store<S>::C densB) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C f[QQ];
  pull<QQ>(A, g, b, 0, sh, f);
  C rR = sum_q<QQ>(f);
  pull<QQ>(A, g, b, 1, sh, f);
  C rB = sum_q<QQ>(f);
  if (rR < C(-10) || rR > C(10) || rB < C(-10) || rB > C(10)) raise_error(err, LBX_DEV_RHO_RANGE, step, cell);
  if (rR < C(0)) rR = C(0);
  if (rB < C(0)) rB = C(0);
  // the phase field the gradient takes (psi_shifted, kernels_fluid_CG.CUF:
  // 728-729: scaled by the fluid densities, 1 and 1 for a single density)
  phi[cell] = (rR / densR - rB / densB) / (rR / densR + rB / densB);
  if (rhoR) { rhoR[2 * size_t(cell)] = rR; rhoB[2 * size_t(cell)] = rB; }
}

// time_step_CG + streaming, two-pass schedule: pull, densities, gradient from
// the phase-field array (DD, two fluid densities: from the density arrays),
// collision, aligned store.
template <typename S, bool DD, int QQ>
__global__ void __launch_bounds__(256) k_cg_collide(const S* __restrict__ A, S* __restrict__ B, Geom g,
                                                     Shift<typename Store<S>::C> sh,
                                                     const typename Store<S>::C* __restrict__ phi,
                                                     const typename Store<S>::C* __restrict__ rhoRa,
                                                     const typename Store<S>::C* __restrict__ rhoBa,
                                                     CGConst<typename Store<S>::C> K) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C fR[QQ], fB[QQ];
  pull<QQ>(A, g, b, 0, sh, fR);
  pull<QQ>(A, g, b, 1, sh, fB);
  C rR = sum_q<QQ>(fR), rB = sum_q<QQ>(fB);
  if (rR < C(0)) rR = C(0);
  if (rB < C(0)) rB = C(0);
  C psix, psiy, psiz;
  if constexpr (DD) {
    // psi from the scaled phase field k_cg_phi stored (the same quotient per
    // neighbour as psi_shifted), the two density gradients from the density
    // arrays
    C psR[3], psB[3], sx, sy, sz;
    grad27(K.L, [&](int dx, int dy, int dz) { return __ldg(phi + at(b, dx, dy, dz)); }, psix, psiy, psiz);
    grad27(K.L, [&](int dx, int dy, int dz) { return __ldg(rhoRa + 2 * size_t(at(b, dx, dy, dz))); }, sx, sy, sz);
    psR[0] = sx; psR[1] = sy; psR[2] = sz;
    grad27(K.L, [&](int dx, int dy, int dz) { return __ldg(rhoBa + 2 * size_t(at(b, dx, dy, dz))); }, sx, sy, sz);
    psB[0] = sx; psB[1] = sy; psB[2] = sz;
    cg_collide_cell_dd<QQ>(K, fR, fB, rR, rB, psix, psiy, psiz, psR, psB);
  } else {
    grad27(K.L, [&](int dx, int dy, int dz) { return __ldg(phi + at(b, dx, dy, dz)); }, psix, psiy, psiz);
    cg_collide_cell<QQ>(K, fR, fB, rR, rB, psix, psiy, psiz);
  }
  store_all<QQ>(B, g, cell, 0, sh, fR);
  store_all<QQ>(B, g, cell, 1, sh, fB);
}

// ---------------------------------------------------------------------------
// Single-pass colour-gradient step.  CTA = TX x TY threads owning the column
// [x0, x0+TX) x [y0, y0+TY) x [z0, z0+ZLEN).  For every plane it computes the
// phase field of the (TX+2) x (TY+2) cells of the column plus its ring from
// the pulled populations into a rolling 4-slot shared window, then collides
// the plane behind it.  The interior threads keep their pulled populations of
// the plane ahead in registers for the next iteration.
// ---------------------------------------------------------------------------
template <int TX, int TY>
struct FusedShape {
  static constexpr int RX = TX + 2, RY = TY + 2, RING = RX * RY, NT = TX * TY;
};

__device__ __forceinline__ int wrapc(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

template <typename S, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_cg_fused(const S* __restrict__ A, S* __restrict__ B, Geom g,
                                                      Shift<typename Store<S>::C> sh,
                                                      CGConst<typename Store<S>::C> K, int zlen,
                                                      unsigned long long* err, int64_t step) {
  using C = typename Store<S>::C;
  using SH = FusedShape<TX, TY>;
  constexpr int NRING = 2 * SH::RX + 2 * TY;  // bottom row, top row, left and right columns
  __shared__ C sphi[4][SH::RING];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * zlen;
  const int zend = min(z0 + zlen, g.nz);
  // every thread computes the phase field of its (wrapped) position, so a
  // partial tile still fills its shared window; only in-range cells collide
  const bool active = (x0 + tx < g.nx) && (y0 + ty < g.ny);
  const int x = wrapc(x0 + tx, g.nx), y = wrapc(y0 + ty, g.ny);

  // phase field of the ring cells of plane z into sphi[slot]
  auto ring_phi = [&](int z, int slot) {
    for (int t = tid; t < NRING; t += SH::NT) {
      int rx, ry;
      if (t < SH::RX) { rx = t; ry = 0; }
      else if (t < 2 * SH::RX) { rx = t - SH::RX; ry = SH::RY - 1; }
      else if (t < 2 * SH::RX + TY) { rx = 0; ry = 1 + t - 2 * SH::RX; }
      else { rx = SH::RX - 1; ry = 1 + t - 2 * SH::RX - TY; }
      Nbr b;
      make_nbr(g, wrapc(x0 + rx - 1, g.nx), wrapc(y0 + ry - 1, g.ny), wrapc(z, g.nz), b);
      C f[Q];
      pull(A, g, b, 0, sh, f);
      C rR = sum_q(f);
      pull(A, g, b, 1, sh, f);
      C rB = sum_q(f);
      if (rR < C(0)) rR = C(0);
      if (rB < C(0)) rB = C(0);
      sphi[slot][ry * SH::RX + rx] = (rR - rB) / (rR + rB);
    }
  };

  C fR[Q], fB[Q];     // populations of the plane being collided
  C nR[Q], nB[Q];     // populations of the plane ahead
  C rRn = 0, rBn = 0; // clamped densities of the plane ahead
  const int own = (ty + 1) * SH::RX + (tx + 1);

  // pull the own cell of plane z into n*, write its phase field to the slot
  auto own_phi = [&](int z, int slot) {
    Nbr b;
    make_nbr(g, x, y, wrapc(z, g.nz), b);
    pull(A, g, b, 0, sh, nR);
    pull(A, g, b, 1, sh, nB);
    C rR = sum_q(nR), rB = sum_q(nB);
    // range check of init_rho*_CG, raised by the CTA that owns the plane
    if (active && z >= z0 && z < zend && (rR < C(-10) || rR > C(10) || rB < C(-10) || rB > C(10)))
      raise_error(err, LBX_DEV_RHO_RANGE, step, at(b, 0, 0, 0));
    if (rR < C(0)) rR = C(0);
    if (rB < C(0)) rB = C(0);
    rRn = rR; rBn = rB;
    sphi[slot][own] = (rR - rB) / (rR + rB);
  };

  // prologue: planes z0-1 and z0
  own_phi(z0 - 1, (z0 + 3) & 3);
  ring_phi(z0 - 1, (z0 + 3) & 3);
  own_phi(z0, z0 & 3);
  ring_phi(z0, z0 & 3);
  for (int z = z0; z < zend; ++z) {
#pragma unroll
    for (int l = 0; l < Q; ++l) { fR[l] = nR[l]; fB[l] = nB[l]; }
    C rR = rRn, rB = rBn;
    own_phi(z + 1, (z + 1) & 3);
    ring_phi(z + 1, (z + 1) & 3);
    __syncthreads();
    if (active) {
      const C* pm = sphi[(z + 3) & 3];
      const C* p0 = sphi[z & 3];
      const C* pp = sphi[(z + 1) & 3];
      C psix, psiy, psiz;
      grad27(K.L,
             [&](int dx, int dy, int dz) {
               const C* pl = dz < 0 ? pm : (dz > 0 ? pp : p0);
               return pl[own + dy * SH::RX + dx];
             },
             psix, psiy, psiz);
      cg_collide_cell(K, fR, fB, rR, rB, psix, psiy, psiz);
      int cell = x + g.nx * (y + g.ny * z);
      store_all(B, g, cell, 0, sh, fR);
      store_all(B, g, cell, 1, sh, fB);
    }
    // The slot read here as plane z-1 is rewritten at iteration z+2 (plane
    // z+3); the barrier of iteration z+1 orders that write after these reads.
  }
}

// init_rho_isfluid_BGK + time_step_BGK + stream_BGK in one pass
template <typename S>
__global__ void __launch_bounds__(256) k_bgk(const S* __restrict__ A, S* __restrict__ B, Geom g,
                                              Shift<typename Store<S>::C> sh, LatticeT<typename Store<S>::C> L,
                                              typename Store<S>::C omega, unsigned long long* err, int64_t step) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C f[Q];
  pull(A, g, b, 0, sh, f);
  C r = sum_q(f);
  if (r < C(-10) || r > C(10)) raise_error(err, LBX_DEV_RHO_RANGE, step, cell);
  const C ONE = 1;
  C invrho = ONE / r;
  C u = invrho * mx(f), v = invrho * my(f), w = invrho * mz(f);
  C usq = L.half_inv_cssq * (u * u + v * v + w * w);
  C omm = ONE - omega;
#pragma unroll
  for (int l = 0; l < Q; ++l) f[l] = f[l] * omm + equil_u(L, r, edot(l, u, v, w), usq, l) * omega;
  store_all(B, g, cell, 0, sh, f);
}

// moments2Fl on the post-streaming populations (pulled from the state)
template <typename S, typename O, int QQ>
__global__ void k_fields(const S* __restrict__ A, const S* Bold, Geom g, int ncomp, Shift<typename Store<S>::C> sh,
                         const int8_t* __restrict__ flags, const int8_t* __restrict__ fold, O* rR, O* rB, O* vel,
                         O* phase) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C fR[QQ], fB[QQ];
  pull_any<QQ>(A, Bold, g, b, 0, sh, fold, fR);
  if (ncomp == 2) pull_any<QQ>(A, Bold, g, b, 1, sh, fold, fB);
  else {
#pragma unroll
    for (int l = 0; l < QQ; ++l) fB[l] = C(0);
  }
  if (sh.split) split_decode<QQ>(C(sh.split[cell]), fR, fB);
  if (sh.sd) sd_to_rb<QQ>(fR, fB);
  C lr = sum_q<QQ>(fR), lb = sum_q<QQ>(fB);
  C rs = lr + lb;
  C inv = C(1) / rs;
  C u = inv * (mx<QQ>(fR) + mx<QQ>(fB)), v = inv * (my<QQ>(fR) + my<QQ>(fB)), w = inv * (mz<QQ>(fR) + mz<QQ>(fB));
  bool ok = (!flags || flags[cell] == LBX_FLUID_FLUID) && rs > C(0);
  if (rR) rR[cell] = ok ? O(lr) : O(0);
  if (rB) rB[cell] = ok ? O(lb) : O(0);
  if (vel) {
    vel[3 * size_t(cell) + 0] = ok ? O(u) : O(0);
    vel[3 * size_t(cell) + 1] = ok ? O(v) : O(0);
    vel[3 * size_t(cell) + 2] = ok ? O(w) : O(0);
  }
  if (phase) phase[cell] = ok ? O((lr - lb) / (lr + lb)) : O(0);
}

template <typename S, int QQ>
__global__ void k_get_pops(const S* __restrict__ A, const S* Bold, Geom g, int ncomp, Shift<typename Store<S>::C> sh,
                           const int8_t* __restrict__ fold, float* pR, float* pB) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C f[QQ];
  if (sh.sd) {  // both halves of each pair are needed for either component
    C f1[QQ];
    pull_any<QQ>(A, Bold, g, b, 0, sh, fold, f);
    pull_any<QQ>(A, Bold, g, b, 1, sh, fold, f1);
    if (sh.split) split_decode<QQ>(C(sh.split[cell]), f, f1);
    sd_to_rb<QQ>(f, f1);
#pragma unroll
    for (int l = 0; l < QQ; ++l) {
      if (pR) pR[size_t(l) * size_t(g.n) + cell] = float(f[l]);
      if (pB) pB[size_t(l) * size_t(g.n) + cell] = float(f1[l]);
    }
    return;
  }
  for (int comp = 0; comp < ncomp; ++comp) {
    float* out = comp ? pB : pR;
    if (!out) continue;
    pull_any<QQ>(A, Bold, g, b, comp, sh, fold, f);
#pragma unroll
    for (int l = 0; l < QQ; ++l) out[size_t(l) * size_t(g.n) + cell] = float(f[l]);
  }
}

// FP64 mass (per component) and momentum of the post-streaming populations,
// block partial sums combined with FP64 atomics.
template <typename S, int QQ>
__global__ void k_sums(const S* __restrict__ A, const S* Bold, Geom g, int ncomp, Shift<typename Store<S>::C> sh,
                       const int8_t* __restrict__ flags, const int8_t* __restrict__ fold, double* out) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  double acc[5] = {0, 0, 0, 0, 0};
  if (x < g.nx && y < g.ny) {
    Nbr b;
    make_nbr(g, x, y, z, b);
    int cell = at(b, 0, 0, 0);
    if (!flags || flags[cell] == LBX_FLUID_FLUID) {
      C f[QQ], f1[QQ];
      if (sh.sd) {
        pull_any<QQ>(A, Bold, g, b, 0, sh, fold, f);
        pull_any<QQ>(A, Bold, g, b, 1, sh, fold, f1);
        if (sh.split) split_decode<QQ>(C(sh.split[cell]), f, f1);
        sd_to_rb<QQ>(f, f1);
      }
      for (int comp = 0; comp < ncomp; ++comp) {
        if (sh.sd) {
          if (comp == 1) {
#pragma unroll
            for (int l = 0; l < QQ; ++l) f[l] = f1[l];
          }
        } else {
          pull_any<QQ>(A, Bold, g, b, comp, sh, fold, f);
        }
        double m = 0;
#pragma unroll
        for (int l = 0; l < QQ; ++l) m += double(f[l]);
        acc[comp] = m;
        acc[2] += double(mx<QQ>(f));
        acc[3] += double(my<QQ>(f));
        acc[4] += double(mz<QQ>(f));
      }
    }
  }
  for (int i = 0; i < 5; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + i, v);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int fluid_alloc(Ctx& c) {
  size_t bytes = size_t(c.ncomp) * size_t(c.q) * size_t(c.n) * c.elem;
  for (int i = 0; i < 2; ++i)
    if (cudaMalloc(&c.pops[i], bytes) != cudaSuccess) return LBX_ERR_ALLOC;
  size_t cb = (c.storage == LBX_STORE_F64) ? 8 : 4;
  if (cudaMalloc(&c.phi, size_t(c.n) * cb) != cudaSuccess) return LBX_ERR_ALLOC;
  // densities interleaved, (rhoR, rhoB) of a cell side by side: one sector
  // per scattered read of both (the sphere kernels read them at the fluid
  // ends of links); rho[1] is rho[0] one element on, both indexed 2 * cell
  if (cudaMalloc(&c.rho[0], 2 * size_t(c.n) * cb) != cudaSuccess) return LBX_ERR_ALLOC;
  c.rho[1] = static_cast<char*>(c.rho[0]) + cb;
  for (int i = 0; i < 2; ++i) {
    if (cudaMalloc(&c.flags[i], size_t(c.n)) != cudaSuccess) return LBX_ERR_ALLOC;
    cudaMemsetAsync(c.flags[i], LBX_FLUID_FLUID, size_t(c.n), c.stream);
  }
  cudaMemsetAsync(c.pops[0], 0, bytes, c.stream);
  cudaMemsetAsync(c.pops[1], 0, bytes, c.stream);
  if (c.sdp)
    for (int i = 0; i < 2; ++i) {
      if (cudaMalloc(&c.split[i], size_t(c.n) * 4) != cudaSuccess) return LBX_ERR_ALLOC;
      cudaMemsetAsync(c.split[i], 0, size_t(c.n) * 4, c.stream);
    }
  return launch_status();
}

void fluid_free(Ctx& c) {
  for (int i = 0; i < 2; ++i) {
    if (c.pops[i]) cudaFree(c.pops[i]);
    if (c.flags[i]) cudaFree(c.flags[i]);
    c.pops[i] = nullptr; c.flags[i] = nullptr;
  }
  if (c.rho[0]) cudaFree(c.rho[0]);  // rho[1] points into it
  c.rho[0] = c.rho[1] = nullptr;
  if (c.phi) cudaFree(c.phi);
  c.phi = nullptr;
  for (int i = 0; i < 2; ++i) {
    if (c.split[i]) cudaFree(c.split[i]);
    c.split[i] = nullptr;
  }
  if (c.lean_plan) cudaFree(c.lean_plan);
  c.lean_plan = nullptr;
}

// fn(std::integral_constant<int, QQ>) with QQ = the context's populations per component
template <typename F>
static int by_lattice(const Ctx& c, F&& fn) {
  if (c.q == Q27) return fn(std::integral_constant<int, Q27>{});
  return fn(std::integral_constant<int, Q>{});
}
static bool two_densities(const Ctx& c) {
  return c.p.model == LBX_MODEL_CG_DIFFDENS || c.p.model == LBX_MODEL_CG_DIFFDENS_D3Q27;
}

static void reset_flags(Ctx& c) {
  for (int i = 0; i < 2; ++i) cudaMemsetAsync(c.flags[i], LBX_FLUID_FLUID, size_t(c.n), c.stream);
  c.fcur = 0;
}

int fluid_set_fields(Ctx& c, const float* d_rR, const float* d_rB, float vx, float vy, float vz) {
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  c.cur = 0;
  reset_flags(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    if (c.sdp)
      k_split_of_fields<<<int((c.n + 255) / 256), 256, 0, c.stream>>>(g, d_rR, d_rB, c.split[0]);
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      if (two_densities(c))
        k_set_fields<S, true, QQ><<<d.grid, d.block, 0, c.stream>>>((S*)c.pops[0], (S*)c.pops[1], g, c.ncomp, d_rR,
                                                                    d_rB, vx, vy, vz, make_cg<C>(c), make_shift<C>(c));
      else
        k_set_fields<S, false, QQ><<<d.grid, d.block, 0, c.stream>>>((S*)c.pops[0], (S*)c.pops[1], g, c.ncomp, d_rR,
                                                                     d_rB, vx, vy, vz, make_cg<C>(c), make_shift<C>(c));
      return launch_status();
    });
  });
}

int fluid_set_pops(Ctx& c, const float* d_pR, const float* d_pB) {
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  c.cur = 0;
  reset_flags(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      if (c.sdp) k_split_of_pops<QQ><<<int((c.n + 255) / 256), 256, 0, c.stream>>>(g, d_pR, d_pB, c.split[0]);
      k_set_pops<S, QQ><<<d.grid, d.block, 0, c.stream>>>((S*)c.pops[0], g, c.ncomp, d_pR, d_pB, make_shift<C>(c));
      return launch_status();
    });
  });
}

void kt_begin(Ctx& c) {
  if (!c.kt_on) return;
  if (c.kt_ev.size() < size_t(2 * (c.kt_n + 1))) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    c.kt_ev.push_back(e0);
    c.kt_ev.push_back(e1);
  }
  cudaEventRecord(c.kt_ev[2 * c.kt_n], c.stream);
}
void kt_end(Ctx& c) {
  if (!c.kt_on) return;
  cudaEventRecord(c.kt_ev[2 * c.kt_n + 1], c.stream);
  c.kt_n += 1;
}

int fluid_init_rho(Ctx& c) {
  if (c.ncomp != 2) return LBX_ERR_STATE;
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      const CGConst<C> K = make_cg<C>(c);
      k_cg_phi<S, QQ><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], g, make_shift<C>(c), (C*)c.phi,
                                                        (C*)c.rho[0], (C*)c.rho[1], c.d_err, c.step + 1, K.densR,
                                                        K.densB);
      return launch_status();
    });
  });
}

int fluid_collide_stream(Ctx& c) {
  if (c.ncomp != 2) return LBX_ERR_STATE;
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    kt_begin(c);
    by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      if (two_densities(c))
        k_cg_collide<S, true, QQ><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], g,
                                                                    make_shift<C>(c), (const C*)c.phi,
                                                                    (const C*)c.rho[0], (const C*)c.rho[1],
                                                                    make_cg<C>(c));
      else
        k_cg_collide<S, false, QQ><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur],
                                                                     g, make_shift<C>(c), (const C*)c.phi, nullptr,
                                                                     nullptr, make_cg<C>(c));
      return 0;
    });
    kt_end(c);
    c.cur = 1 - c.cur;
    return launch_status();
  });
}

// column shape of the single-pass kernel
constexpr int FTX = 32, FTY = 8;

static int fused_zlen(const Ctx& c) {
  // enough z-segments to give every SM a few CTAs; longer columns amortise
  // the two extra planes each segment recomputes
  long cols = long((c.nx + FTX - 1) / FTX) * long((c.ny + FTY - 1) / FTY);
  long target = 148L * 4;
  long segs = (target + cols - 1) / cols;
  if (segs < 1) segs = 1;
  int zlen = int((c.nz + segs - 1) / segs);
  if (zlen < 4) zlen = (c.nz < 4) ? c.nz : 4;
  return zlen;
}

int fluid_fused(Ctx& c) {
  Geom g = geom(c);
  int zlen = fused_zlen(c);
  dim3 block(FTX, FTY, 1);
  dim3 grid((c.nx + FTX - 1) / FTX, (c.ny + FTY - 1) / FTY, (c.nz + zlen - 1) / zlen);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    kt_begin(c);
    k_cg_fused<S, FTX, FTY><<<grid, block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], g,
                                                          make_shift<C>(c), make_cg<C>(c), zlen, c.d_err,
                                                          c.step + 1);
    kt_end(c);
    c.cur = 1 - c.cur;
    return launch_status();
  });
}

int fluid_bgk(Ctx& c) {
  if (c.ncomp != 1) return LBX_ERR_STATE;
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    kt_begin(c);
    k_bgk<S><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], g, make_shift<C>(c),
                                               make_lattice<C>(), C(1) / C(c.p.tau), c.d_err, c.step + 1);
    kt_end(c);
    c.cur = 1 - c.cur;
    return launch_status();
  });
}

int fluid_step(Ctx& c) {
  int rc;
  if (c.ncomp == 1) {
    rc = fluid_bgk(c);
  } else if (c.fused == 2) {
    rc = fluid_lean(c);
  } else if (c.fused == 1) {
    rc = fluid_fused(c);
  } else {
    rc = fluid_init_rho(c);
    if (!rc) rc = fluid_collide_stream(c);
  }
  if (!rc) c.step += 1;
  return rc;
}

// flags of the particle path for readback: the mask of the last step and the
// dead-source flags of the pull (nullptr without particles)
int particles_flags_slot(const Ctx& c);
int particles_active(const Ctx& c);
static const int8_t* mask_flags(const Ctx& c) { return particles_active(c) ? c.flags[particles_flags_slot(c)] : nullptr; }
static const int8_t* dead_flags(const Ctx& c) { return particles_active(c) ? c.flags[c.fcur] : nullptr; }

int fluid_get_fields(Ctx& c, void* rR, void* rB, void* vel, void* phase, int f64) {
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    const S* A = (const S*)c.pops[c.cur];
    const S* Bo = (const S*)c.pops[1 - c.cur];
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      if (f64)
        k_fields<S, double, QQ><<<d.grid, d.block, 0, c.stream>>>(A, Bo, g, c.ncomp, make_shift<C>(c), mask_flags(c),
                                                                  dead_flags(c), (double*)rR, (double*)rB,
                                                                  (double*)vel, (double*)phase);
      else
        k_fields<S, float, QQ><<<d.grid, d.block, 0, c.stream>>>(A, Bo, g, c.ncomp, make_shift<C>(c), mask_flags(c),
                                                                 dead_flags(c), (float*)rR, (float*)rB, (float*)vel,
                                                                 (float*)phase);
      return launch_status();
    });
  });
}

int fluid_get_pops(Ctx& c, float* pR, float* pB) {
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      k_get_pops<S, QQ><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (const S*)c.pops[1 - c.cur], g,
                                                          c.ncomp, make_shift<C>(c), dead_flags(c), pR, pB);
      return launch_status();
    });
  });
}

int fluid_get_sums(Ctx& c, double* d_out5) {
  LaunchDims d = cell_dims(c);
  Geom g = geom(c);
  cudaMemsetAsync(d_out5, 0, 5 * sizeof(double), c.stream);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    return by_lattice(c, [&](auto qt) {
      constexpr int QQ = decltype(qt)::value;
      k_sums<S, QQ><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (const S*)c.pops[1 - c.cur], g,
                                                      c.ncomp, make_shift<C>(c), mask_flags(c), dead_flags(c), d_out5);
      return launch_status();
    });
  });
}

}  // namespace lbx
