// lbx_device.cuh — device helpers shared by the fluid and particle kernels:
// periodic neighbour indexing, pull gathers, the equilibrium, the
// colour-gradient collision of one cell and the host-side constant builders.
#pragma once
#include <type_traits>

#include "lbx_common.cuh"
#include "lbx_ctx.h"

namespace lbx {

// ---------------------------------------------------------------------------
// indexing
// ---------------------------------------------------------------------------
struct Nbr {
  int x, xm, xp;  // column index and its periodic neighbours
  int ry[3];      // ny-row offsets (y-1, y, y+1) * nx
  int rz[3];      // plane offsets (z-1, z, z+1) * nx * ny
};

__device__ __forceinline__ void make_nbr(const Geom& g, int x, int y, int z, Nbr& b) {
  b.x = x;
  b.xm = (x == 0) ? g.nx - 1 : x - 1;
  b.xp = (x == g.nx - 1) ? 0 : x + 1;
  int ym = (y == 0) ? g.ny - 1 : y - 1, yp = (y == g.ny - 1) ? 0 : y + 1;
  int zm = (z == 0) ? g.nz - 1 : z - 1, zp = (z == g.nz - 1) ? 0 : z + 1;
  b.ry[0] = ym * g.nx; b.ry[1] = y * g.nx; b.ry[2] = yp * g.nx;
  const int plane = g.nx * g.ny;
  b.rz[0] = zm * plane; b.rz[1] = z * plane; b.rz[2] = zp * plane;
}

// linear index of x + (dx,dy,dz), periodic
__device__ __forceinline__ int at(const Nbr& b, int dx, int dy, int dz) {
  int xx = dx == 0 ? b.x : (dx > 0 ? b.xp : b.xm);
  return xx + b.ry[dy + 1] + b.rz[dz + 1];
}

// e_l . (u,v,w) with the zero components dropped, summed in x,y,z order
template <typename C>
__device__ __forceinline__ C edot(int l, C u, C v, C w) {
  C s = C(0);
  bool any = false;
  if (ex(l)) { s = ex(l) > 0 ? u : -u; any = true; }
  if (ey(l)) { s = any ? (ey(l) > 0 ? s + v : s - v) : (ey(l) > 0 ? v : -v); any = true; }
  if (ez(l)) { s = any ? (ez(l) > 0 ? s + w : s - w) : (ez(l) > 0 ? w : -w); any = true; }
  return s;
}

// equil, kernels_fluid_CG.CUF:30-38, with the velocity-square term hoisted
template <typename C>
__device__ __forceinline__ C equil_u(const LatticeT<C>& L, C rho, C edu, C usq_term, int l) {
  C uv = L.inv_cssq * edu;
  return rho * L.w[wclass27(l)] * (C(1) + uv + C(0.5) * (uv * uv) - usq_term);
}

// gather the post-streaming populations of one component (pull of the push
// streaming of stream*_CG + halo pushes)
template <int QQ = Q, typename S, typename C>
__device__ __forceinline__ void pull(const S* __restrict__ A, const Geom& g, const Nbr& b, int comp,
                                     const Shift<C>& sh, C* f) {
#pragma unroll
  for (int l = 0; l < QQ; ++l) f[l] = Store<S>::ld(A + pidx(g, comp, l, at(b, -ex(l), -ey(l), -ez(l))), sh.at(comp, l));
}

template <int QQ = Q, typename S, typename C>
__device__ __forceinline__ void store_all(S* __restrict__ B, const Geom& g, int cell, int comp, const Shift<C>& sh,
                                          const C* f) {
#pragma unroll
  for (int l = 0; l < QQ; ++l) Store<S>::st(B + pidx(g, comp, l, cell), f[l], sh.at(comp, l));
}

// The post-streaming populations of a cell, pulled from the post-collision
// state A; a spheredead source (flags of the previous step) leaves the
// destination's stale value, which is B's entry.
template <int QQ = Q, typename S, typename C>
__device__ __forceinline__ void pull_dead(const S* __restrict__ A, const S* Bold, const Geom& g, const Nbr& b,
                                          int comp, const Shift<C>& sh, const int8_t* __restrict__ fold, C* f) {
  const int self = at(b, 0, 0, 0);
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    int src = at(b, -ex(l), -ey(l), -ez(l));
    if (l > 0 && fold[src] == LBX_FLUID_SPHEREDEAD)
      f[l] = Store<S>::ld(Bold + pidx(g, comp, l, self), sh.at(comp, l));
    else
      f[l] = Store<S>::ld(A + pidx(g, comp, l, src), sh.at(comp, l));
  }
}

// pull_dead when the flags of the previous step are given, plain pull otherwise
template <int QQ = Q, typename S, typename C>
__device__ __forceinline__ void pull_any(const S* __restrict__ A, const S* Bold, const Geom& g, const Nbr& b,
                                         int comp, const Shift<C>& sh, const int8_t* __restrict__ fold, C* f) {
  if (fold) pull_dead<QQ>(A, Bold, g, b, comp, sh, fold, f);
  else pull<QQ>(A, g, b, comp, sh, f);
}

// Sum / difference pairs (Shift::sd): what the per-component pulls gave
// (R + B and R - B, shifts removed) into the components, and back before
// the per-component stores.
template <int QQ = Q, typename C>
__device__ __forceinline__ void sd_to_rb(C* f0, C* f1) {
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    const C s = f0[l], d = f1[l];
    f0[l] = C(0.5) * (s + d);
    f1[l] = C(0.5) * (s - d);
  }
}
// Sum / predicted-split pairs: the pulled (total, E) pairs of a cell back to
// (total, R - B) with the phase field ph the pairs were encoded against.
template <int QQ = Q, typename C>
__device__ __forceinline__ void split_decode(C ph, const C* f0, C* f1) {
#pragma unroll
  for (int l = 0; l < QQ; ++l) f1[l] = f1[l] + ph * f0[l];
}
template <int QQ = Q, typename C>
__device__ __forceinline__ void rb_to_sd(C* f0, C* f1) {
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    const C r = f0[l], b = f1[l];
    f0[l] = r + b;
    f1[l] = r - b;
  }
}

template <int QQ = Q, typename C>
__device__ __forceinline__ C sum_q(const C* f) {
  C r = f[0];
#pragma unroll
  for (int l = 1; l < QQ; ++l) r = r + f[l];
  return r;
}
// manual_u/v/w sums, kernels_fluid_CG.CUF:511-529 (without the 1/rho factor)
// (D3Q27: the same sums continued over the corners 19..26 in increasing l,
// kernels_fluid_CG.CUF:511-523)
template <int QQ, typename C>
__device__ __forceinline__ C msum_q(const C* q, int axis) {
  C s = C(0);
  bool any = false;
#pragma unroll
  for (int l = 1; l < QQ; ++l) {
    const int e = axis == 0 ? ex(l) : (axis == 1 ? ey(l) : ez(l));
    if (!e) continue;
    s = any ? (e > 0 ? s + q[l] : s - q[l]) : (e > 0 ? q[l] : -q[l]);
    any = true;
  }
  return s;
}
template <int QQ = Q, typename C> __device__ __forceinline__ C mx(const C* q) {
  if constexpr (QQ == Q) return q[1] - q[2] + q[7] - q[8] - q[9] + q[10] + q[11] - q[12] - q[13] + q[14];
  else return msum_q<QQ>(q, 0);
}
template <int QQ = Q, typename C> __device__ __forceinline__ C my(const C* q) {
  if constexpr (QQ == Q) return q[3] - q[4] + q[7] - q[8] + q[9] - q[10] + q[15] - q[16] - q[17] + q[18];
  else return msum_q<QQ>(q, 1);
}
template <int QQ = Q, typename C> __device__ __forceinline__ C mz(const C* q) {
  if constexpr (QQ == Q) return q[5] - q[6] + q[11] - q[12] + q[13] - q[14] + q[15] - q[16] + q[17] - q[18];
  else return msum_q<QQ>(q, 2);
}

// Constants of the colour-gradient collision, derived on the host like
// SetConstants (main.CUF:1043-1162).
template <typename C>
struct CGConst {
  LatticeT<C> L;
  C inv_viscR, inv_viscB;  // 1/viscR, 1/viscB
  C sigma, beta;
  // two fluid densities (the DIFFDENS build): densR_d, densB_d, alphaCG_d and
  // the phi / varphi / psi / xi tables per weight class (dimensions_m.CUF:231-261)
  C densR, densB;
  C alpha[2];
  C phi[4], varphi[4], psi[4], xi[4];
};

// equilCG, kernels_fluid_CG.CUF:40-49 (component k = 0 R, 1 B), with the
// velocity-square term hoisted like equil_u
template <typename C>
__device__ __forceinline__ C equil_cg(const CGConst<C>& K, C rho, C edu, C usq_term, int k, int l) {
  const C uv = K.L.inv_cssq * edu;
  const int c = wclass27(l);
  return rho * (K.phi[c] + K.varphi[c] * K.alpha[k] + K.L.w[c] * (uv + C(0.5) * (uv * uv) - usq_term));
}

// ---------------------------------------------------------------------------
// time_step_CG at one fluid cell (kernels_fluid_CG.CUF:689-846).  fR/fB hold
// the post-streaming populations on entry and the post-collision ones on exit.
// rhoR/rhoB are the clamped densities of init_rho*_CG, psi the colour
// gradient (HIGHGRAD, D3Q27 weights).
// ---------------------------------------------------------------------------
template <int QQ = Q, typename C>
__device__ __forceinline__ void cg_collide_cell(const CGConst<C>& K, C* fR, C* fB, C rhoR, C rhoB, C psix,
                                                C psiy, C psiz) {
  const C ONE = 1, HALF = C(0.5);
  const LatticeT<C>& L = K.L;
  C rhosum = rhoR + rhoB;
  C phase_field = (rhoR - rhoB) / (rhoR + rhoB);
  C viscavg = ONE / (HALF * (ONE + phase_field) * K.inv_viscR + HALF * (ONE - phase_field) * K.inv_viscB);
  C omega = ONE / (viscavg / L.cssq + HALF);
  C omm = ONE - omega;
  C invrho = ONE / rhosum;
  C u = invrho * mx<QQ>(fR) + invrho * mx<QQ>(fB);
  C v = invrho * my<QQ>(fR) + invrho * my<QQ>(fB);
  C w = invrho * mz<QQ>(fR) + invrho * mz<QQ>(fB);
  C usq = L.half_inv_cssq * (u * u + v * v + w * w);
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    C e = edot(l, u, v, w);
    fR[l] = fR[l] * omm + equil_u(L, rhoR, e, usq, l) * omega;
    fB[l] = fB[l] * omm + equil_u(L, rhoB, e, usq, l) * omega;
  }
  C psinorm_sq = psix * psix + psiy * psiy + psiz * psiz;
  if (psinorm_sq > C(1.e-20)) {
    C psinorm = sqrt(psinorm_sq);
    C inv_psq = ONE / psinorm_sq;
    C acoeff = C(9) / C(4) * omega * K.sigma;
    C kR = rhoR * invrho, kB = rhoB * invrho;
    C coef = K.beta * rhoR * rhoB * (invrho * invrho);
    C inv_t1 = ONE / psinorm;                 // rec_fact = 1
    C inv_t2 = ONE / (L.rec[2] * psinorm);    // rec_fact = sqrt(2)
    C inv_t3 = ONE / (L.rec[3] * psinorm);    // rec_fact = sqrt(3) (D3Q27 corners)
#pragma unroll
    for (int l = 0; l < QQ; ++l) {
      C edp = edot(l, psix, psiy, psiz);
      C temp = psinorm * (L.w[wclass27(l)] * (edp * edp) * inv_psq - L.b[wclass27(l)]);
      C fd = fR[l] + fB[l] + acoeff * temp;
      C feq = rhoR * L.w[wclass27(l)] + rhoB * L.w[wclass27(l)];
      C cosphi;
      if (l == 0) cosphi = C(0);
      else {
        C t1 = L.rec[wclass27(l)] * psinorm;
        cosphi = (t1 <= C(1.e-20)) ? C(0) : edp * (wclass27(l) == 1 ? inv_t1 : (wclass27(l) == 2 ? inv_t2 : inv_t3));
      }
      C t = coef * cosphi;
      fR[l] = fd * kR + t * feq;
      fB[l] = fd * kB - t * feq;
    }
  }
}

// time_step_CG of the DIFFDENS build at one fluid cell (kernels_fluid_CG.CUF:
// 689-837 with DIFFDENS): the phase field scaled by the fluid densities, the
// BGK step towards equilCG plus the viscous correction
//   viscavg (psi_l u.grad(rho_k) + xi_l (G_k : e_l e_l)),  G_k = u grad(rho_k)^T + its transpose,
// and the recolouring weighted by equilCG at rest.  psR / psB: D3Q27
// gradients of the two densities; psi: gradient of the scaled phase field.
template <int QQ = Q, typename C>
__device__ __forceinline__ void cg_collide_cell_dd(const CGConst<C>& K, C* fR, C* fB, C rhoR, C rhoB, C psix,
                                                   C psiy, C psiz, const C psR[3], const C psB[3]) {
  const C ONE = 1, HALF = C(0.5), ZERO = 0;
  const LatticeT<C>& L = K.L;
  C rhosum = rhoR + rhoB;
  C phase_field = (rhoR / K.densR - rhoB / K.densB) / (rhoR / K.densR + rhoB / K.densB);
  C viscavg = ONE / (HALF * (ONE + phase_field) * K.inv_viscR + HALF * (ONE - phase_field) * K.inv_viscB);
  C omega = ONE / (viscavg / L.cssq + HALF);
  C omm = ONE - omega;
  C invrho = ONE / rhosum;
  C u = invrho * mx<QQ>(fR) + invrho * mx<QQ>(fB);
  C v = invrho * my<QQ>(fR) + invrho * my<QQ>(fB);
  C w = invrho * mz<QQ>(fR) + invrho * mz<QQ>(fB);
  C usq = L.half_inv_cssq * (u * u + v * v + w * w);
  const C vpR = u * psR[0] + v * psR[1] + w * psR[2];  // dot_product(myvel, psi_R)
  const C vpB = u * psB[0] + v * psB[1] + w * psB[2];
  const C uu[3] = {u, v, w};
  C gR[3], gB[3];  // diagonal of tensor_product + its transpose
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    gR[i] = uu[i] * psR[i] + uu[i] * psR[i];
    gB[i] = uu[i] * psB[i] + uu[i] * psB[i];
  }
#pragma unroll
  for (int l = 0; l < QQ; ++l) {
    const int c = wclass27(l);
    const C e = edot(l, u, v, w);
    const C cx = C(ex(l) * ex(l)), cy = C(ey(l) * ey(l)), cz = C(ez(l) * ez(l));  // cmat_d(i,i,l)
    const C tR = gR[0] * cx + gR[1] * cy + gR[2] * cz;
    const C tB = gB[0] * cx + gB[1] * cy + gB[2] * cz;
    fR[l] = fR[l] * omm + (equil_cg(K, rhoR, e, usq, 0, l) + viscavg * (K.psi[c] * vpR + K.xi[c] * tR)) * omega;
    fB[l] = fB[l] * omm + (equil_cg(K, rhoB, e, usq, 1, l) + viscavg * (K.psi[c] * vpB + K.xi[c] * tB)) * omega;
  }
  C psinorm_sq = psix * psix + psiy * psiy + psiz * psiz;
  if (psinorm_sq > C(1.e-20)) {
    C psinorm = sqrt(psinorm_sq);
    C inv_psq = ONE / psinorm_sq;
    C acoeff = C(9) / C(4) * omega * K.sigma;
    C kR = rhoR * invrho, kB = rhoB * invrho;
    C coef = K.beta * rhoR * rhoB * (invrho * invrho);
    C inv_t1 = ONE / psinorm;
    C inv_t2 = ONE / (L.rec[2] * psinorm);
    C inv_t3 = ONE / (L.rec[3] * psinorm);
#pragma unroll
    for (int l = 0; l < QQ; ++l) {
      C edp = edot(l, psix, psiy, psiz);
      C temp = psinorm * (L.w[wclass27(l)] * (edp * edp) * inv_psq - L.b[wclass27(l)]);
      C fd = fR[l] + fB[l] + acoeff * temp;
      C feq = equil_cg(K, rhoR, ZERO, ZERO, 0, l) + equil_cg(K, rhoB, ZERO, ZERO, 1, l);
      C cosphi;
      if (l == 0) cosphi = C(0);
      else {
        C t1 = L.rec[wclass27(l)] * psinorm;
        cosphi = (t1 <= C(1.e-20)) ? C(0) : edp * (wclass27(l) == 1 ? inv_t1 : (wclass27(l) == 2 ? inv_t2 : inv_t3));
      }
      C t = coef * cosphi;
      fR[l] = fd * kR + t * feq;
      fB[l] = fd * kB - t * feq;
    }
  }
}

// DIFFDENS gradients from the neighbours' densities (rho_at returns the pair
// (rhoR, rhoB) of neighbour (dx, dy, dz)): psi of the scaled phase field and
// the gradients of the two densities (kernels_fluid_CG.CUF:720-741)
template <typename C, typename F>
__device__ __forceinline__ void grad27_dd(const CGConst<C>& K, F&& rho_at, C& psix, C& psiy, C& psiz, C psR[3],
                                          C psB[3]) {
  psix = C(0); psiy = C(0); psiz = C(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) psR[i] = psB[i] = C(0);
#pragma unroll
  for (int l = 1; l < Q27; ++l) {
    C rs, bs;
    rho_at(ex27(l), ey27(l), ez27(l), rs, bs);
    const C ps = (rs / K.densR - bs / K.densB) / (rs / K.densR + bs / K.densB);
    const C a = K.L.a27[wclass27(l)];
    if (ex27(l)) {
      const C ax = ex27(l) > 0 ? a : -a;
      psix = psix + ax * ps;
      psR[0] = psR[0] + ax * rs;
      psB[0] = psB[0] + ax * bs;
    }
    if (ey27(l)) {
      const C ay = ey27(l) > 0 ? a : -a;
      psiy = psiy + ay * ps;
      psR[1] = psR[1] + ay * rs;
      psB[1] = psB[1] + ay * bs;
    }
    if (ez27(l)) {
      const C az = ez27(l) > 0 ? a : -a;
      psiz = psiz + az * ps;
      psR[2] = psR[2] + az * rs;
      psB[2] = psB[2] + az * bs;
    }
  }
}

// colour gradient psi = sum_l a27_l e_l phi(x + e_l), l = 1..26 in reference order
template <typename C, typename F>
__device__ __forceinline__ void grad27(const LatticeT<C>& L, F&& phi_at, C& psix, C& psiy, C& psiz) {
  psix = C(0); psiy = C(0); psiz = C(0);
#pragma unroll
  for (int l = 1; l < Q27; ++l) {
    C ps = phi_at(ex27(l), ey27(l), ez27(l));
    C a = L.a27[wclass27(l)];
    if (ex27(l)) psix = psix + (ex27(l) > 0 ? a : -a) * ps;
    if (ey27(l)) psiy = psiy + (ey27(l) > 0 ? a : -a) * ps;
    if (ez27(l)) psiz = psiz + (ez27(l) > 0 ? a : -a) * ps;
  }
}


// ---------------------------------------------------------------------------
// launch geometry and host-side constant builders
// ---------------------------------------------------------------------------
struct LaunchDims {
  dim3 grid, block;
};

inline LaunchDims cell_dims(const Ctx& c) {
  int bx = (c.nx % 128 == 0) ? 128 : ((c.nx % 64 == 0) ? 64 : 32);
  int by = 256 / bx;
  LaunchDims d;
  d.block = dim3(bx, by, 1);
  d.grid = dim3((c.nx + bx - 1) / bx, (c.ny + by - 1) / by, c.nz);
  return d;
}

template <typename C>
inline Shift<C> make_shift(const Ctx& c) {
  Shift<C> s;
  LatticeT<C> L = make_lattice<C>(c.q);
  bool shifted = c.storage != LBX_STORE_F32 && c.storage != LBX_STORE_F64;
  float r0[2] = {c.p.rho0R, c.p.rho0B};
  s.sd = c.sd ? 1 : 0;
  // sum / difference pairs: the shifts of R + B and of R - B (the predicted
  // split's deviation E is stored unshifted)
  if (c.sd) {
    r0[0] = c.p.rho0R + c.p.rho0B;
    r0[1] = c.sdp ? 0.0f : c.p.rho0R - c.p.rho0B;
  }
  s.split = c.sdp ? c.split[c.cur] : nullptr;
  for (int comp = 0; comp < 2; ++comp)
    for (int k = 0; k < 4; ++k) s.s[comp][k] = shifted ? C(L.w[k] * C(r0[comp])) : C(0);
  return s;
}

template <typename C>
inline CGConst<C> make_cg(const Ctx& c) {
  CGConst<C> K;
  K.L = make_lattice<C>(c.q);
  const C HALF = C(0.5);
  C viscR = K.L.cssq * (C(c.p.tauR) - HALF);  // SetConstants, main.CUF:1069-1070
  C viscB = K.L.cssq * (C(c.p.tauB) - HALF);
  K.inv_viscR = C(1) / viscR;
  K.inv_viscB = C(1) / viscB;
  K.sigma = C(c.p.sigma);
  K.beta = C(c.p.beta);
  // DIFFDENS constants (SetConstants, main.CUF:1047-1083; dimensions_m.CUF:231-261)
  const bool dd = c.p.model == LBX_MODEL_CG_DIFFDENS || c.p.model == LBX_MODEL_CG_DIFFDENS_D3Q27;
  const C ONE = C(1), TWO = C(2), FOUR = C(4), FIVE = C(5), SIX = C(6), EIGHT = C(8), TWELVE = C(12),
          TWENTYFOUR = C(24);
  K.densR = dd ? C(c.p.densR) : ONE;
  K.densB = dd ? C(c.p.densB) : ONE;
  const C p0 = K.L.w[0];
  if (K.densR == ONE) {
    K.alpha[0] = p0;
    K.alpha[1] = (-ONE + K.alpha[0]) * (K.densR / K.densB) + ONE;
  } else {  // as the reference writes it (not (1 - alpha_B) densB / densR)
    K.alpha[1] = p0;
    K.alpha[0] = (ONE / (-ONE + K.alpha[1])) * (K.densB / K.densR) + ONE;
  }
  if (c.q == Q27) {  // dimensions_m.CUF:145-191
    const C NINE = C(9), THREE = C(3);
    K.phi[0] = C(0); K.phi[1] = TWO / C(19.0); K.phi[2] = ONE / C(38.0); K.phi[3] = ONE / C(152.0);
    K.varphi[0] = ONE; K.varphi[1] = -TWO / C(19.0); K.varphi[2] = -ONE / C(38.0); K.varphi[3] = -ONE / C(152.0);
    K.psi[0] = C(-20.0) / NINE; K.psi[1] = -TWO / NINE; K.psi[2] = ONE / C(36.0); K.psi[3] = ONE / C(36.0);
    K.xi[0] = C(0); K.xi[1] = ONE / THREE; K.xi[2] = ONE / TWELVE; K.xi[3] = ONE / C(48.0);
  } else {
    K.phi[0] = C(0); K.phi[1] = ONE / TWELVE; K.phi[2] = ONE / TWENTYFOUR; K.phi[3] = C(0);
    K.varphi[0] = ONE; K.varphi[1] = -ONE / TWELVE; K.varphi[2] = -ONE / TWENTYFOUR; K.varphi[3] = C(0);
    K.psi[0] = -FIVE / TWO; K.psi[1] = -ONE / SIX; K.psi[2] = ONE / TWENTYFOUR; K.psi[3] = C(0);
    K.xi[0] = C(0); K.xi[1] = ONE / FOUR; K.xi[2] = ONE / EIGHT; K.xi[3] = C(0);
  }
  return K;
}

inline Geom geom(const Ctx& c) { return Geom{c.nx, c.ny, c.nz, c.n, c.ncomp}; }

template <typename F>
inline int by_storage(const Ctx& c, F&& fn) {
  switch (c.storage) {
    case LBX_STORE_F32: return fn((float*)nullptr);
    case LBX_STORE_F16:
    case LBX_STORE_F16_SD:
    case LBX_STORE_F16_SDP: return fn((__half*)nullptr);
    case LBX_STORE_BF16:
    case LBX_STORE_BF16_SD:
    case LBX_STORE_BF16_SDP: return fn((__nv_bfloat16*)nullptr);
    case LBX_STORE_F64: return fn((double*)nullptr);
  }
  return LBX_ERR_ARG;
}

inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : LBX_ERR_CUDA;
}


}  // namespace lbx
