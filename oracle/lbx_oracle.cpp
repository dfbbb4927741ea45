/*
 * lbx_oracle.cpp — CPU restatement of the LBcuda per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker of the CUDA
 * path and the CPU baseline timed beside it.  Only tests/, the smoke check
 * and the bench's cpu_baseline / reference arm may load it; the product
 * library never links or calls it.
 *
 * PARITY UNPINNED: the reference (CUDA Fortran, copmat/LBcuda) needs
 * nvfortran + MPI, neither of which exists where this was written, and the
 * reference ships no golden outputs or known-answer tests (its Tests/ holds
 * input decks only).  This restatement therefore follows the reference source
 * line by line (citations below, paths relative to the reference project)
 * and is checked against analytic invariants in tests/, not against outputs
 * of the reference itself.
 *
 * Structure mirrors the reference on purpose: arrays carry the 1-cell halo
 * ring (0..n+1), the periodic wrap is the halo copy of fixPeriodic
 * (main.CUF:577-1000), collision is in place (time_step_CG) and streaming is
 * the push of stream*_CG plus the halo pushes of stream_CG_x/_y/_z.  That
 * keeps it independent of the GPU design (SoA without halo, pull streaming,
 * in-kernel wrap) that it checks.
 *
 * Templated on the fluid type T and the particle type P:
 *   mode 0: T=float,  P=float   — the reference's own precision
 *   mode 1: T=float,  P=double  — FP32 fluid with FP64 particle state
 *   mode 2: T=double, P=double  — FP64 everything (error reference)
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/lbx.h"

namespace {

constexpr int Q = 19;
constexpr int Q27 = 27;

/* ---- lattice tables, dimensions_m.CUF:201-300 (D3Q19, noD3Q27) ------------- */
/* directions 0..18 are D3Q19; the D3Q27 build (dimensions_m.CUF:117-198)
 * appends the eight corners 19..26 in the same table order */
const int EX[Q27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
const int EY[Q27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1};
const int EZ[Q27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};
/* D3Q27 neighbour set used by HIGHGRAD and the belts, dimensions_m.CUF:275-281 */
const int EX27[Q27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
const int EY27[Q27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1};
const int EZ27[Q27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};

/* weight class of direction l: number of non-zero components (0..3) */
inline int wcls(int l) { return (l == 0) ? 0 : (l <= 6 ? 1 : (l <= 18 ? 2 : 3)); }

template <typename T>
struct Tables {
  T p[Q27], b_l[Q27], rec_fact[Q27], a27[Q27], p27[Q27];
  T phi[Q27], varphi[Q27], psi[Q27], xi[Q27]; /* DIFFDENS tables */
  T cssq;
  int q; /* 19 or 27 populations */
  explicit Tables(int nq = Q) : q(nq) {
    /* all arithmetic in T, in the order the Fortran parameter expressions use */
    const T ONE = 1, TWO = 2, THREE = 3, SIX = 6, TWELVE = 12, TWENTYFOUR = 24;
    const T FOUR = 4, FIVE = 5, EIGHT = 8, NINE = 9, TEN = 10, TWENTYSEVEN = 27, FIFTYFOUR = 54;
    cssq = T(1.0) / T(3.0);                                   /* dimensions_m.CUF:94 */
    const T q0 = (TWO / THREE) * (TWO / THREE) * (TWO / THREE);   /* :283-286 */
    const T q1 = (TWO / THREE) * (TWO / THREE) * (ONE / SIX);
    const T q2 = (ONE / SIX) * (ONE / SIX) * (TWO / THREE);
    const T q3 = (ONE / SIX) * (ONE / SIX) * (ONE / SIX);
    T pc[4], bc[4], phc[4], vpc[4], psc[4], xc[4];
    if (q == Q) { /* D3Q19, :201-261 */
      pc[0] = T(1.0) / T(3.0); pc[1] = T(1.0) / T(18.0); pc[2] = T(1.0) / T(36.0); pc[3] = 0;
      const T b_xi = T(0.5);                                  /* Leclaire, :222 */
      bc[0] = -(TWO + TWO * b_xi) / (THREE * b_xi + TWELVE);
      bc[1] = (b_xi) / (SIX * b_xi + TWENTYFOUR);
      bc[2] = ONE / (SIX * b_xi + TWENTYFOUR);
      bc[3] = 0;
      phc[0] = T(0); phc[1] = ONE / TWELVE; phc[2] = ONE / TWENTYFOUR; phc[3] = 0;
      vpc[0] = ONE; vpc[1] = -ONE / TWELVE; vpc[2] = -ONE / TWENTYFOUR; vpc[3] = 0;
      psc[0] = -FIVE / TWO; psc[1] = -ONE / SIX; psc[2] = ONE / TWENTYFOUR; psc[3] = 0;
      xc[0] = T(0); xc[1] = ONE / FOUR; xc[2] = ONE / EIGHT; xc[3] = 0;
    } else {      /* D3Q27, :117-198 */
      pc[0] = q0; pc[1] = q1; pc[2] = q2; pc[3] = q3;
      bc[0] = -(TEN / TWENTYSEVEN); bc[1] = TWO / TWENTYSEVEN; bc[2] = ONE / FIFTYFOUR; bc[3] = ONE / T(216.0);
      phc[0] = T(0); phc[1] = TWO / T(19.0); phc[2] = ONE / T(38.0); phc[3] = ONE / T(152.0);
      vpc[0] = ONE; vpc[1] = -TWO / T(19.0); vpc[2] = -ONE / T(38.0); vpc[3] = -ONE / T(152.0);
      psc[0] = T(-20.0) / NINE; psc[1] = -TWO / NINE; psc[2] = ONE / T(36.0); psc[3] = ONE / T(36.0);
      xc[0] = T(0); xc[1] = ONE / THREE; xc[2] = ONE / TWELVE; xc[3] = ONE / T(48.0);
    }
    for (int l = 0; l < Q27; ++l) {
      const int c = wcls(l);
      p[l] = pc[c];
      b_l[l] = bc[c];
      phi[l] = phc[c];
      varphi[l] = vpc[c];
      psi[l] = psc[c];
      xi[l] = xc[c];
      rec_fact[l] = std::sqrt(T(EX[l] * EX[l] + EY[l] * EY[l] + EZ[l] * EZ[l])); /* SetConstants, main.CUF:1098 */
      T w = (l == 0) ? q0 : (l <= 6 ? q1 : (l <= 18 ? q2 : q3));
      p27[l] = w;
      a27[l] = (l == 0) ? T(0) : w / cssq;                        /* :292-298 */
    }
  }
};

/* equil, kernels_fluid_CG.CUF:30-38 */
template <typename T>
inline T equil(const Tables<T>& tb, T rho, T u, T v, T w, int l) {
  const T ONE = 1, HALF = T(0.5);
  T uv = (ONE / tb.cssq) * (u * T(EX[l]) + v * T(EY[l]) + w * T(EZ[l]));
  return rho * tb.p[l] * (ONE + uv + HALF * (uv * uv) - (HALF / tb.cssq) * (u * u + v * v + w * w));
}

/* equilCG, kernels_fluid_CG.CUF:40-49 (alpha = alphaCG_d(k)) */
template <typename T>
inline T equil_cg(const Tables<T>& tb, T rho, T u, T v, T w, T alpha, int l) {
  const T HALF = T(0.5);
  T uv = (T(1) / tb.cssq) * (u * T(EX[l]) + v * T(EY[l]) + w * T(EZ[l]));
  return rho * (tb.phi[l] + tb.varphi[l] * alpha + tb.p[l] * (uv + HALF * (uv * uv) - (HALF / tb.cssq) * (u * u + v * v + w * w)));
}

template <typename T>
inline T nint_t(T x) { return std::round(x); } /* Fortran NINT: half away from zero */

struct Particle;

template <typename T, typename P>
class Oracle {
 public:
  lbx_params prm;
  int nx, ny, nz, sx, sy, sz;  /* interior and padded sizes */
  int64_t ncell_pad;
  Tables<T> tb;
  int q = Q; /* populations per component: 19, or 27 for the D3Q27 models */
  int model;
  int flip = 0;  /* 0-based reference `flipflop - 1` */
  int64_t step = 0;
  /* pops[c][buf][l*ncell_pad + idx] */
  std::vector<T> pops[2][2];
  std::vector<T> rho[2];      /* rhoR_d, rhoB_d */
  std::vector<int8_t> flags[2];
  int err_code = 0, err_step = 0;
  int64_t err_where = 0;
  /* physical constants as the reference derives them (SetConstants) */
  T viscR, viscB, omega_bgk;
  bool diffdens = false; /* LBX_MODEL_CG_DIFFDENS: the reference's DIFFDENS build */
  T densR = 1, densB = 1, alphaCG[2] = {0, 0};

  Oracle(const lbx_params& p) : prm(p) {
    nx = p.nx; ny = p.ny; nz = p.nz;
    q = (p.model == LBX_MODEL_CG_D3Q27 || p.model == LBX_MODEL_CG_DIFFDENS_D3Q27) ? Q27 : Q;
    tb = Tables<T>(q);
    sx = nx + 2; sy = ny + 2; sz = nz + 2;
    ncell_pad = int64_t(sx) * sy * sz;
    model = p.model;
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    for (int c = 0; c < ncomp; ++c)
      for (int b = 0; b < 2; ++b) pops[c][b].assign(size_t(q) * ncell_pad, T(0));
    for (int c = 0; c < 2; ++c) rho[c].assign(ncell_pad, T(0));
    for (int b = 0; b < 2; ++b) flags[b].assign(ncell_pad, int8_t(LBX_FLUID_FLUID));
    const T HALF = T(0.5);
    viscR = tb.cssq * (T(p.tauR) - HALF); /* main.CUF:1069-1071 */
    viscB = tb.cssq * (T(p.tauB) - HALF);
    omega_bgk = T(1) / T(p.tau);
    /* SetConstants, main.CUF:1047-1083 */
    diffdens = (model == LBX_MODEL_CG_DIFFDENS || model == LBX_MODEL_CG_DIFFDENS_D3Q27);
    const T ONE = 1;
    densR = diffdens ? T(p.densR) : ONE;
    densB = diffdens ? T(p.densB) : ONE;
    if (densR == ONE) {
      alphaCG[0] = tb.p[0];
      alphaCG[1] = (-ONE + alphaCG[0]) * (densR / densB) + ONE;
    } else {
      alphaCG[1] = tb.p[0];
      alphaCG[0] = (ONE / (-ONE + alphaCG[1])) * (densB / densR) + ONE;
    }
  }

  inline int64_t id(int i, int j, int k) const { return i + int64_t(sx) * (j + int64_t(sy) * k); }
  inline T& f(int c, int b, int l, int64_t idx) { return pops[c][b][size_t(l) * ncell_pad + idx]; }

  void raise(int code, int64_t where) {
#pragma omp critical(orc_err)
    {
      if (!err_code) { err_code = code; err_step = int(step); err_where = where; }
    }
  }

  /* ---- periodic halo (fixPeriodic / bc_per_*2 / bc_edge_*2 / isfluid_per_*2) ----
   * Every halo cell (faces, edges and corners) receives the periodic image of
   * an interior cell, for the populations l = 1..Q-1 (faiPops), the two
   * density arrays (faiRho) or the flags. */
  inline int wrapi(int i, int n) const { return i < 1 ? i + n : (i > n ? i - n : i); }
  template <typename F>
  void for_halo(F&& fn) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < sz; ++k)
      for (int j = 0; j < sy; ++j)
        for (int i = 0; i < sx; ++i) {
          if (i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nz) continue;
          fn(id(i, j, k), id(wrapi(i, nx), wrapi(j, ny), wrapi(k, nz)));
        }
  }
  void halo_pops(int b) {
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    for_halo([&](int64_t h, int64_t s) {
      for (int c = 0; c < ncomp; ++c)
        for (int l = 1; l < q; ++l) f(c, b, l, h) = f(c, b, l, s);
    });
  }
  void halo_rho() {
    for_halo([&](int64_t h, int64_t s) { rho[0][h] = rho[0][s]; rho[1][h] = rho[1][s]; });
  }
  void halo_flags(int b) {
    for_halo([&](int64_t h, int64_t s) { flags[b][h] = flags[b][s]; });
  }

  /* ---- initial conditions: setupPops, kernels_fluid_CG.CUF:313-346 ------------- */
  void set_fields(const float* rR, const float* rB, float vx, float vy, float vz) {
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    flip = 0;
    step = 0;
    for (int c = 0; c < ncomp; ++c)
      for (int b = 0; b < 2; ++b) std::fill(pops[c][b].begin(), pops[c][b].end(), T(0));
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          int64_t x = id(i, j, k);
          T r0 = T(rR[h]);
          T r1 = (ncomp == 2 && rB) ? T(rB[h]) : T(0);
          rho[0][x] = r0;
          rho[1][x] = r1;
          for (int l = 0; l < q; ++l) {
            if (diffdens) { /* setup2, kernels_fluid_CG.CUF:176-178 */
              f(0, 0, l, x) = equil_cg(tb, r0, T(vx), T(vy), T(vz), alphaCG[0], l);
              f(1, 0, l, x) = equil_cg(tb, r1, T(vx), T(vy), T(vz), alphaCG[1], l);
              continue;
            }
            f(0, 0, l, x) = equil(tb, r0, T(vx), T(vy), T(vz), l);
            if (ncomp == 2) f(1, 0, l, x) = equil(tb, r1, T(vx), T(vy), T(vz), l);
          }
          flags[0][x] = LBX_FLUID_FLUID;
          flags[1][x] = LBX_FLUID_FLUID;
        }
    halo_pops(0);
    halo_rho();
    halo_flags(0);
    halo_flags(1);
    last_flags = 0;
  }

  void set_pops(const float* pR, const float* pB) {
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    flip = 0;
    step = 0;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          int64_t x = id(i, j, k);
          for (int l = 0; l < q; ++l) {
            f(0, 0, l, x) = T(pR[h + n * l]);
            if (ncomp == 2) f(1, 0, l, x) = pB ? T(pB[h + n * l]) : T(0);
          }
          flags[0][x] = LBX_FLUID_FLUID;
          flags[1][x] = LBX_FLUID_FLUID;
        }
    halo_pops(0);
    halo_flags(0);
    halo_flags(1);
  }

  /* ---- init_rhoR_CG / init_rhoB_CG, kernels_fluid_CG.CUF:398-509 ------------- */
  void init_rho() {
    const T minRho = T(-10), maxRho = T(10), MINDENS = T(0);
    const int b = flip;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          for (int c = 0; c < 2; ++c) {
            if (flags[b][x] == LBX_FLUID_FLUID) {
              T r = f(c, b, 0, x);
              for (int l = 1; l < q; ++l) r = r + f(c, b, l, x); /* fixed order 0..18 */
              if (r < minRho || r > maxRho) raise(LBX_DEV_RHO_RANGE, (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1)));
              if (r < MINDENS) r = MINDENS;
              rho[c][x] = r;
            } else {
              rho[c][x] = MINDENS;
            }
          }
        }
    halo_rho(); /* fixPeriodic(.false., .true.) */
  }

  /* manual_u/v/w, kernels_fluid_CG.CUF:511-529 */
  /* sum_l e_l,d f_l over the nonzero components in increasing l (the
   * left-to-right order of manual_u/v/w, kernels_fluid_CG.CUF:511-529, and
   * of the D3Q27 sums there); from zero, so the first term enters exactly */
  T msum(const T* f_, const int* e) const {
    T s = 0;
    for (int l = 1; l < q; ++l) {
      if (e[l] > 0) s = s + f_[l];
      else if (e[l] < 0) s = s - f_[l];
    }
    return s;
  }
  T mom_x(const T* f_, T inv) const { return inv * msum(f_, EX); }
  T mom_y(const T* f_, T inv) const { return inv * msum(f_, EY); }
  T mom_z(const T* f_, T inv) const { return inv * msum(f_, EZ); }

  /* ---- time_step_CG, kernels_fluid_CG.CUF:531-848 (HIGHGRAD; DIFFDENS when
   * the model is LBX_MODEL_CG_DIFFDENS) --------------------------------------- */
  void time_step_cg() {
    const T ONE = 1, HALF = T(0.5), ZERO = 0, NINE = 9, FOUR = 4;
    const T mylimit = T(1.e-20);
    const T sigma = T(prm.sigma), beta = T(prm.beta);
    const int b = flip;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          if (flags[b][x] != LBX_FLUID_FLUID) continue;
          T tR[Q27], tB[Q27], fd[Q27];
          for (int l = 0; l < q; ++l) { tR[l] = f(0, b, l, x); tB[l] = f(1, b, l, x); }
          T rhoR = rho[0][x], rhoB = rho[1][x];
          T rhosum = rhoR + rhoB;
          T phase_field = (rhoR / densR - rhoB / densB) / (rhoR / densR + rhoB / densB);
          T viscavg = ONE / (HALF * (ONE + phase_field) * (ONE / viscR) + HALF * (ONE - phase_field) * (ONE / viscB));
          T omega = ONE / (viscavg / tb.cssq + HALF);
          T oneminusomega = ONE - omega;
          T invrho = ONE / rhosum;
          T u = mom_x(tR, invrho) + mom_x(tB, invrho);
          T v = mom_y(tR, invrho) + mom_y(tB, invrho);
          T w = mom_z(tR, invrho) + mom_z(tB, invrho);
          T psix = ZERO, psiy = ZERO, psiz = ZERO;
          T psR[3] = {ZERO, ZERO, ZERO}, psB[3] = {ZERO, ZERO, ZERO};
          for (int l = 1; l < Q27; ++l) { /* HIGHGRAD, :720-741 */
            int64_t y = id(i + EX27[l], j + EY27[l], k + EZ27[l]);
            T rs = rho[0][y], bs = rho[1][y];
            T ps = (rs / densR - bs / densB) / (rs / densR + bs / densB);
            psix = psix + tb.a27[l] * T(EX27[l]) * ps;
            psiy = psiy + tb.a27[l] * T(EY27[l]) * ps;
            psiz = psiz + tb.a27[l] * T(EZ27[l]) * ps;
            if (diffdens) {
              psR[0] = psR[0] + tb.a27[l] * T(EX27[l]) * rs;
              psR[1] = psR[1] + tb.a27[l] * T(EY27[l]) * rs;
              psR[2] = psR[2] + tb.a27[l] * T(EZ27[l]) * rs;
              psB[0] = psB[0] + tb.a27[l] * T(EX27[l]) * bs;
              psB[1] = psB[1] + tb.a27[l] * T(EY27[l]) * bs;
              psB[2] = psB[2] + tb.a27[l] * T(EZ27[l]) * bs;
            }
          }
          if (diffdens) { /* :743-786 */
            const T vel[3] = {u, v, w};
            T vR = vel[0] * psR[0] + vel[1] * psR[1] + vel[2] * psR[2];
            T vB = vel[0] * psB[0] + vel[1] * psB[1] + vel[2] * psB[2];
            T gR[3], gB[3]; /* diagonal of tensor_product(myvel, psi) + transpose */
            for (int d = 0; d < 3; ++d) {
              gR[d] = vel[d] * psR[d] + vel[d] * psR[d];
              gB[d] = vel[d] * psB[d] + vel[d] * psB[d];
            }
            for (int l = 0; l < q; ++l) {
              const T cm[3] = {T(EX[l] * EX[l]), T(EY[l] * EY[l]), T(EZ[l] * EZ[l])}; /* cmat_d(d,d,l) */
              T tc = gR[0] * cm[0] + gR[1] * cm[1] + gR[2] * cm[2];
              tR[l] = tR[l] * oneminusomega +
                      (equil_cg(tb, rhoR, u, v, w, alphaCG[0], l) + viscavg * (tb.psi[l] * vR + tb.xi[l] * tc)) * omega;
            }
            for (int l = 0; l < q; ++l) {
              const T cm[3] = {T(EX[l] * EX[l]), T(EY[l] * EY[l]), T(EZ[l] * EZ[l])};
              T tc = gB[0] * cm[0] + gB[1] * cm[1] + gB[2] * cm[2];
              tB[l] = tB[l] * oneminusomega +
                      (equil_cg(tb, rhoB, u, v, w, alphaCG[1], l) + viscavg * (tb.psi[l] * vB + tb.xi[l] * tc)) * omega;
            }
          } else {
            for (int l = 0; l < q; ++l) tR[l] = tR[l] * oneminusomega + equil(tb, rhoR, u, v, w, l) * omega;
            for (int l = 0; l < q; ++l) tB[l] = tB[l] * oneminusomega + equil(tb, rhoB, u, v, w, l) * omega;
          }
          T psinorm_sq = psix * psix + psiy * psiy + psiz * psiz;
          if (psinorm_sq > mylimit) { /* perturbation + recolouring, :803-837 */
            T psinorm = std::sqrt(psinorm_sq);
            T acoeff = NINE / FOUR * omega * sigma;
            for (int l = 0; l < q; ++l) {
              T edp = T(EX[l]) * psix + T(EY[l]) * psiy + T(EZ[l]) * psiz;
              T temp = psinorm * (tb.p[l] * (edp * edp) / psinorm_sq - tb.b_l[l]);
              fd[l] = tR[l] + tB[l] + acoeff * temp;
            }
            for (int l = 0; l < q; ++l) {
              T feq = diffdens ? equil_cg(tb, rhoR, ZERO, ZERO, ZERO, alphaCG[0], l) +
                                     equil_cg(tb, rhoB, ZERO, ZERO, ZERO, alphaCG[1], l)
                               : equil(tb, rhoR, ZERO, ZERO, ZERO, l) + equil(tb, rhoB, ZERO, ZERO, ZERO, l);
              T edp = T(EX[l]) * psix + T(EY[l]) * psiy + T(EZ[l]) * psiz;
              T temp1 = tb.rec_fact[l] * psinorm;
              T cosphi = (temp1 <= mylimit) ? ZERO : edp / temp1;
              T temp = beta * rhoR * rhoB * cosphi / (rhosum * rhosum);
              f(0, b, l, x) = fd[l] * rhoR / rhosum + temp * feq;
              f(1, b, l, x) = fd[l] * rhoB / rhosum - temp * feq;
            }
          } else {
            for (int l = 0; l < q; ++l) { f(0, b, l, x) = tR[l]; f(1, b, l, x) = tB[l]; }
          }
        }
    halo_pops(b); /* fixPeriodic(.true., .false.) */
  }

  /* ---- init_rho_isfluid_BGK + time_step_BGK, kernels_fluid_BGK.CUF:205-256 --- */
  void time_step_bgk() {
    const T ONE = 1;
    const T omega = omega_bgk, oneminusomega = ONE - omega;
    const int b = flip;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          if (flags[b][x] != LBX_FLUID_FLUID) { rho[0][x] = 0; continue; }
          T q[Q];
          for (int l = 0; l < Q; ++l) q[l] = f(0, b, l, x);
          T r = q[0];
          for (int l = 1; l < Q; ++l) r = r + q[l];
          if (r < T(-10) || r > T(10)) raise(LBX_DEV_RHO_RANGE, (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1)));
          rho[0][x] = r;
          T invrho = ONE / r;
          T u = mom_x(q, invrho), v = mom_y(q, invrho), w = mom_z(q, invrho);
          for (int l = 0; l < Q; ++l) f(0, b, l, x) = q[l] * oneminusomega + equil(tb, r, u, v, w, l) * omega;
        }
    halo_pops(b); /* periodic wrap of the post-collision populations */
  }

  /* ---- flipflop*Pop0_CG + stream*_CG + stream_CG_x/_y/_z, CG.CUF:851-1141 ---- */
  void stream() {
    const int b = flip, o = 1 - flip;
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    /* interior pushes; each target is written by exactly one source, so the
     * k-parallel loop is race-free */
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          for (int c = 0; c < ncomp; ++c) f(c, o, 0, x) = f(c, b, 0, x);
          if (flags[b][x] == LBX_FLUID_SPHEREDEAD) continue;
          for (int c = 0; c < ncomp; ++c)
            for (int l = 1; l < q; ++l) f(c, o, l, id(i + EX[l], j + EY[l], k + EZ[l])) = f(c, b, l, x);
        }
    /* halo cells push into the interior (stream_CG_x, _y, _z) */
    auto halo_push = [&](int i, int j, int k) {
      int64_t x = id(i, j, k);
      if (flags[b][x] == LBX_FLUID_SPHEREDEAD) return;
      for (int l = 1; l < q; ++l) {
        int i1 = i + EX[l], j1 = j + EY[l], k1 = k + EZ[l];
        if (1 <= i1 && i1 <= nx && 1 <= j1 && j1 <= ny && 1 <= k1 && k1 <= nz)
          for (int c = 0; c < ncomp; ++c) f(c, o, l, id(i1, j1, k1)) = f(c, b, l, x);
      }
    };
    for (int k = 0; k < sz; ++k)
      for (int j = 0; j < sy; ++j) { halo_push(0, j, k); halo_push(nx + 1, j, k); }
    for (int k = 0; k < sz; ++k)
      for (int i = 0; i < sx; ++i) { halo_push(i, 0, k); halo_push(i, ny + 1, k); }
    for (int j = 0; j < sy; ++j)
      for (int i = 0; i < sx; ++i) { halo_push(i, j, 0); halo_push(i, j, nz + 1); }
  }

  /* =====================================================================
   * Particles (PARTICLES build), kernels_fluid_PART.CUF and main.CUF.
   * pos[slot][13*i + c]: c = 0..2 x, 3..5 v, 6..8 omega (body frame),
   * 9..12 quaternion; force[slot][12*i + c]: 0..2 total force, 3..5 bounce-back
   * force, 6..8 total torque, 9..11 bounce-back torque (dimensions_m.CUF:352-360).
   * ===================================================================== */
  int np = 0;
  bool lrotate = false;
  std::vector<P> pos[2], force[2];
  std::vector<double> myf, myf2, myt, myt2;
  std::vector<int> partVol, oldpartVol;
  int rmin = 0, rmax = 0, sphereMax = 0;
  std::vector<int8_t> issub;   /* (2rmax+1)^3, index (i+rmax) + w*((j+rmax) + w*(k+rmax)) */
  std::vector<int> owner;      /* debugfluid_d: 1-based particle index, 0 = none */
  static constexpr int TX = 8, TY = 4, TZ = 4; /* defines.h:14-22 tile */
  int nbx = 0, nby = 0, nbz = 0;
  std::vector<std::vector<int>> tiles;          /* matrixAtoms_d / dim_matAtm_d */
  P rdim;
  T buz;

  int tw() const { return 2 * rmax + 1; }
  int8_t sub(int i, int j, int k) const { return issub[(i + rmax) + tw() * ((j + rmax) + tw() * (k + rmax))]; }
  P& ps(int slot, int i, int c) { return pos[slot][13 * size_t(i) + c]; }
  P& fa(int slot, int i, int c) { return force[slot][12 * size_t(i) + c]; }

  /* spherical_template, main.CUF:1990-2130 */
  void spherical_template() {
    const P sqrcut = rdim * rdim;
    rmin = int(std::floor(rdim));
    rmax = int(rdim + P(1));
    int w = tw();
    issub.assign(size_t(w) * w * w, int8_t(LBX_FLUID_FLUID));
    auto at = [&](int i, int j, int k) -> int8_t& { return issub[(i + rmax) + w * ((j + rmax) + w * (k + rmax))]; };
    for (int k = -rmax; k <= rmax; ++k)
      for (int j = -rmax; j <= rmax; ++j)
        for (int i = -rmax; i <= rmax; ++i)
          if (P(i * i + j * j + k * k) <= sqrcut) at(i, j, k) = LBX_FLUID_SPHEREDEAD;
    for (int k = -rmin; k <= rmin; ++k)
      for (int j = -rmin; j <= rmin; ++j)
        for (int i = -rmin; i <= rmin; ++i)
          if (at(i, j, k) == LBX_FLUID_SPHEREDEAD)
            for (int l = 1; l < Q; ++l)
              if (at(i + EX[l], j + EY[l], k + EZ[l]) == LBX_FLUID_FLUID) { at(i, j, k) = LBX_FLUID_SPHERELIST; break; }
    at(0, 0, 0) = LBX_FLUID_PARTICLECM;
    sphereMax = rmax * rmax;
  }

  /* getDeltai/j/k, kernels_fluid_PART.CUF:182-228 */
  int getDelta(int i, int c, int n) const {
    int d = i - c;
    if (P(c) - rdim < P(1) || P(c) + rdim > P(n)) {
      if (P(c) + rdim > P(n) && P(i) < rdim) d = i - c + n;
      else if (P(c) - rdim < P(1) && P(i) > P(n) - rdim) d = i - c - n;
    }
    return d;
  }
  int nintp(P x) const { return int(std::round(x)); }

  /* zeroListAtomsGPU + makeListAtomsGPU, kernels_fluid_PART.CUF:2315-2451, in
   * particle-index order (the reference's atomic order is not deterministic) */
  void make_lists(int slot) {
    for (auto& t : tiles) t.clear();
    for (int l = 0; l < np; ++l) {
      P x = ps(slot, l, 0), y = ps(slot, l, 1), z = ps(slot, l, 2);
      int ci[3] = {int(std::ceil(x)), int(std::ceil(y)), int(std::ceil(z))};
      P xc[3] = {x, y, z};
      int nn[3] = {nx, ny, nz};
      int td[3] = {TX, TY, TZ};
      int box[3][4];
      for (int d = 0; d < 3; ++d) {
        if (!prm.exact_tiles) {
          /* every cell of the template box [nint - rmax, nint + rmax], split at
           * the periodic edge (the reference's box, int(x +- rdim), misses
           * template cells for integer radii) */
          int c0 = nintp(xc[d]) - rmax, c1 = nintp(xc[d]) + rmax;
          if (c0 < 1) { box[d][0] = 1; box[d][1] = c1; box[d][2] = c0 + nn[d]; box[d][3] = nn[d]; }
          else if (c1 > nn[d]) { box[d][0] = 1; box[d][1] = c1 - nn[d]; box[d][2] = c0; box[d][3] = nn[d]; }
          else { box[d][0] = c0; box[d][1] = c1; box[d][2] = td[d]; box[d][3] = -td[d]; }
          continue;
        }
        box[d][0] = int(xc[d] - rdim); /* real -> integer truncation */
        box[d][1] = int(xc[d] + rdim);
        if (box[d][0] < 1) {
          box[d][0] = 1; box[d][1] = int(P(ci[d]) + rdim); box[d][2] = int(P(ci[d]) - rdim + P(nn[d])); box[d][3] = nn[d];
        } else if (box[d][1] > nn[d]) {
          box[d][0] = 1; box[d][1] = int(P(ci[d]) + rdim - P(nn[d])); box[d][2] = int(P(ci[d]) - rdim); box[d][3] = nn[d];
        } else {
          box[d][2] = td[d]; box[d][3] = -td[d];
        }
      }
      for (int lk = 0; lk < 2; ++lk) {
        int mink = (box[2][2 * lk] - 1) / TZ + 1, maxk = (box[2][2 * lk + 1] - 1) / TZ + 1;
        for (int k = mink; k <= maxk; ++k) {
          if (k < 1 || k > nbz) continue;
          for (int lj = 0; lj < 2; ++lj) {
            int minj = (box[1][2 * lj] - 1) / TY + 1, maxj = (box[1][2 * lj + 1] - 1) / TY + 1;
            for (int j = minj; j <= maxj; ++j) {
              if (j < 1 || j > nby) continue;
              for (int li = 0; li < 2; ++li) {
                int mini = (box[0][2 * li] - 1) / TX + 1, maxi = (box[0][2 * li + 1] - 1) / TX + 1;
                for (int i = mini; i <= maxi; ++i) {
                  if (i < 1 || i > nbx) continue;
                  auto& t = tiles[(i - 1) + size_t(nbx) * ((j - 1) + size_t(nby) * (k - 1))];
                  if (int(t.size()) >= 1000) raise(LBX_DEV_LIST_OVERFLOW, l);
                  else t.push_back(l);
                }
              }
            }
          }
        }
      }
    }
  }
  const std::vector<int>& tile_of(int i, int j, int k) const {
    return tiles[(i - 1) / TX + size_t(nbx) * ((j - 1) / TY + size_t(nby) * ((k - 1) / TZ))];
  }

  /* init_isfluid_CG + setmyfluid, kernels_fluid_PART.CUF:85-117,230-264 */
  void init_isfluid(int b) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          owner[x] = 0;
          bool updated = false;
          for (int a : tile_of(i, j, k)) {
            if (updated) break;
            int di = getDelta(i, nintp(ps(b, a, 0)), nx), dj = getDelta(j, nintp(ps(b, a, 1)), ny),
                dk = getDelta(k, nintp(ps(b, a, 2)), nz);
            if (std::abs(di) <= rmax && std::abs(dj) <= rmax && std::abs(dk) <= rmax) {
              int8_t v = sub(di, dj, dk);
              if (v != LBX_FLUID_FLUID) {
                updated = true;
                flags[b][x] = v;
#pragma omp atomic
                partVol[a] += 1;
                owner[x] = a + 1;
              }
            }
          }
          if (!updated) flags[b][x] = LBX_FLUID_FLUID;
        }
    halo_flags(b);
  }

  bool particle_moved(int a) {
    return nintp(ps(0, a, 0)) != nintp(ps(1, a, 0)) || nintp(ps(0, a, 1)) != nintp(ps(1, a, 1)) ||
           nintp(ps(0, a, 2)) != nintp(ps(1, a, 2));
  }

  /* min-image offset of a cell from a particle, scaled to length rdim
   * (the rtemp/rversor blocks of del_fluid, make_fluid and the bounce-back) */
  void lever(int i, int j, int k, int a, int b, bool image, P r[3]) {
    r[0] = P(i) - ps(b, a, 0);
    r[1] = P(j) - ps(b, a, 1);
    r[2] = P(k) - ps(b, a, 2);
    if (image) {
      const P aaa = P(1) / P(nx), bbb = P(1) / P(ny), ccc = P(1) / P(nz);
      r[0] = r[0] - P(nx) * P(nintp(aaa * r[0]));
      r[1] = r[1] - P(ny) * P(nintp(bbb * r[1]));
      r[2] = r[2] - P(nz) * P(nintp(ccc * r[2]));
    }
    P modr = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int d = 0; d < 3; ++d) r[d] = rdim / modr * r[d];
  }

  template <typename A, typename B>
  static void cross3(const A a[3], const B b[3], P out[3]) {
    out[0] = P(a[1]) * P(b[2]) - P(a[2]) * P(b[1]);
    out[1] = P(a[2]) * P(b[0]) - P(a[0]) * P(b[2]);
    out[2] = P(a[0]) * P(b[1]) - P(a[1]) * P(b[0]);
  }

  void add_acc(std::vector<double>& acc, int a, const double v[3]) {
    for (int d = 0; d < 3; ++d) {
#pragma omp atomic
      acc[3 * size_t(a) + d] += v[d];
    }
  }

  /* del_fluid, kernels_fluid_PART.CUF:383-561 */
  void del_fluid(int b, int a, int i, int j, int k) {
    const int o = 1 - b;
    int di = getDelta(i, nintp(ps(o, a, 0)), nx), dj = getDelta(j, nintp(ps(o, a, 1)), ny),
        dk = getDelta(k, nintp(ps(o, a, 2)), nz);
    if (di * di + dj * dj + dk * dk > sphereMax) return;
    int64_t x = id(i, j, k);
    int8_t fo = flags[o][x], fn = flags[b][x];
    if (fo != LBX_FLUID_FLUID || (fn != LBX_FLUID_SPHERELIST && fn != LBX_FLUID_SPHEREDEAD)) return;
    T rR = rho[0][x], rB = rho[1][x];
    T rhosum = rR + rB, invrho = T(1) / rhosum;
    T qR[Q], qB[Q];
    for (int l = 0; l < Q; ++l) { qR[l] = f(0, b, l, x); qB[l] = f(1, b, l, x); }
    T u = mom_x(qR, invrho) + mom_x(qB, invrho);
    T v = mom_y(qR, invrho) + mom_y(qB, invrho);
    T w = mom_z(qR, invrho) + mom_z(qB, invrho);
    T ft[3] = {(rR + rB) * u, (rR + rB) * v, (rR + rB) * w};
    double acc[3] = {double(ft[0]), double(ft[1]), double(ft[2])};
    add_acc(myf2, a, acc);
    if (lrotate) {
      P r[3], t[3];
      /* the spheredead branch of the reference skips the minimum image */
      lever(i, j, k, a, b, fn == LBX_FLUID_SPHERELIST, r);
      cross3(r, ft, t);
      double tt[3] = {double(t[0]), double(t[1]), double(t[2])};
      add_acc(myt2, a, tt);
    }
  }

  /* compute_onebelt_density_twofluids / compute_secbelt_density_twofluids,
   * kernels_fluid_PART.CUF:783-862 */
  int onebelt(int b, int i, int j, int k, T& Rs, T& Bs) {
    Rs = 0; Bs = 0;
    int D = 0;
    for (int l = 1; l < Q27; ++l) {
      int64_t y = id(i + EX27[l], j + EY27[l], k + EZ27[l]);
      if (flags[b][y] == LBX_FLUID_FLUID && flags[1 - b][y] == LBX_FLUID_FLUID) {
        Rs = Rs + rho[0][y]; Bs = Bs + rho[1][y]; D += 1;
      }
    }
    if (D) { Rs = Rs / T(D); Bs = Bs / T(D); }
    return D;
  }
  int secbelt(int b, int i, int j, int k, T& Rs, T& Bs) {
    Rs = 0; Bs = 0;
    int D = 0;
    for (int kk = -2; kk <= 2; ++kk)
      for (int jj = -2; jj <= 2; ++jj)
        for (int ii = -2; ii <= 2; ++ii) {
          if (!(ii == -2 || ii == 2 || jj == -2 || jj == 2 || kk == -2 || kk == 2)) continue;
          int i1 = (i + ii + nx - 1) % nx + 1, j1 = (j + jj + ny - 1) % ny + 1, k1 = (k + kk + nz - 1) % nz + 1;
          int64_t y = id(i1, j1, k1);
          if (flags[b][y] == LBX_FLUID_FLUID && flags[1 - b][y] == LBX_FLUID_FLUID) {
            Rs = Rs + rho[0][y]; Bs = Bs + rho[1][y]; D += 1;
          }
        }
    if (D) { Rs = Rs / T(D); Bs = Bs / T(D); }
    return D;
  }

  /* make_fluid + initialize_newnode_fluids, kernels_fluid_PART.CUF:563-747,896-913 */
  void make_fluid(int b, int a, int i, int j, int k) {
    const int o = 1 - b;
    int di = getDelta(i, nintp(ps(o, a, 0)), nx), dj = getDelta(j, nintp(ps(o, a, 1)), ny),
        dk = getDelta(k, nintp(ps(o, a, 2)), nz);
    if (di * di + dj * dj + dk * dk > sphereMax) return;
    int64_t x = id(i, j, k);
    int8_t fo = flags[o][x], fn = flags[b][x];
    if ((fo != LBX_FLUID_SPHERELIST && fo != LBX_FLUID_SPHEREDEAD) || fn != LBX_FLUID_FLUID) return;
    T Rs, Bs;
    if (onebelt(b, i, j, k, Rs, Bs) == 0)
      if (secbelt(b, i, j, k, Rs, Bs) == 0) { /* fix_onebelt_density_twofluids: empty */ }
    T u = T(ps(b, a, 3)), v = T(ps(b, a, 4)), w = T(ps(b, a, 5));
    rho[0][x] = Rs;
    rho[1][x] = Bs;
    for (int l = 0; l < Q; ++l) {
      f(0, b, l, x) = equil(tb, Rs, u, v, w, l);
      f(1, b, l, x) = equil(tb, Bs, u, v, w, l);
    }
    T ft[3] = {-(Rs + Bs) * u, -(Rs + Bs) * v, -(Rs + Bs) * w};
    double acc[3] = {double(ft[0]), double(ft[1]), double(ft[2])};
    add_acc(myf2, a, acc);
    if (lrotate) {
      P r[3], t[3];
      lever(i, j, k, a, b, fo == LBX_FLUID_SPHERELIST, r);
      cross3(r, ft, t);
      double tt[3] = {double(t[0]), double(t[1]), double(t[2])};
      add_acc(myt2, a, tt);
    }
  }

  template <typename F>
  void for_cells_with_tile_atoms(F&& fn) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          for (int a : tile_of(i, j, k)) fn(a, i, j, k);
  }

  /* quaternion helpers, kernels_fluid_PART.CUF:1830-1871 */
  static void qmult(const P a[4], const P b[4], P o[4]) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    P c[3];
    c[0] = a[2] * b[3] - a[3] * b[2];
    c[1] = a[3] * b[1] - a[1] * b[3];
    c[2] = a[1] * b[2] - a[2] * b[1];
    for (int d = 0; d < 3; ++d) o[d + 1] = a[0] * b[d + 1] + b[0] * a[d + 1] + c[d];
  }
  static void qtrimult(const P a[4], const P b[4], const P c[4], P o[4]) {
    P t[4];
    qmult(b, c, t);
    qmult(a, t, o);
  }
  /* body vector -> lab frame, q (0,v) q* */
  void to_lab(int b, int a, const P v[3], P out[3]) {
    P q[4] = {ps(b, a, 9), ps(b, a, 10), ps(b, a, 11), ps(b, a, 12)};
    P qc[4] = {q[0], -q[1], -q[2], -q[3]};
    P qv[4] = {P(0), v[0], v[1], v[2]};
    P o[4];
    qtrimult(q, qv, qc, o);
    out[0] = o[1]; out[1] = o[2]; out[2] = o[3];
  }

  /* compute_virtual_rho (Janus), kernels_fluid_PART.CUF:299-352 */
  void virtual_rho_janus(int b) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          if (flags[b][x] != LBX_FLUID_SPHERELIST) continue;
          int a = owner[x] - 1;
          P r[3] = {P(i) - ps(b, a, 0), P(j) - ps(b, a, 1), P(k) - ps(b, a, 2)};
          const P aaa = P(1) / P(nx), bbb = P(1) / P(ny), ccc = P(1) / P(nz);
          r[0] = r[0] - P(nx) * P(nintp(aaa * r[0]));
          r[1] = r[1] - P(ny) * P(nintp(bbb * r[1]));
          r[2] = r[2] - P(nz) * P(nintp(ccc * r[2]));
          P modr = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
          for (int d = 0; d < 3; ++d) r[d] = r[d] / modr;
          P ax[3] = {P(1), P(0), P(0)}, xl[3];
          to_lab(b, a, ax, xl);
          P c = xl[0] * r[0] + xl[1] * r[1] + xl[2] * r[2];
          if (c < P(0)) { rho[0][x] = 0; rho[1][x] = 1; }
          else { rho[0][x] = 1; rho[1][x] = 0; }
        }
  }

  /* compute_densities_wall + compute_onebelt_density_2fl_weights,
   * kernels_fluid_PART.CUF:267-297,864-894 (neutral wetting) */
  void virtual_rho_neutral(int b) {
    std::vector<T> nR(ncell_pad), nB(ncell_pad);
    std::vector<char> set(ncell_pad, 0);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          int8_t fl = flags[b][x];
          if (fl != LBX_FLUID_WALL && fl != LBX_FLUID_SPHERELIST) continue;
          T Rs = 0, Bs = 0, Ds = 0;
          for (int l = 1; l < Q27; ++l) {
            int64_t y = id(i + EX27[l], j + EY27[l], k + EZ27[l]);
            if (flags[b][y] == LBX_FLUID_FLUID) {
              Rs = Rs + tb.p27[l] * rho[0][y]; Bs = Bs + tb.p27[l] * rho[1][y]; Ds = Ds + tb.p27[l];
            }
          }
          if (Ds != T(0)) { Rs = Rs / Ds; Bs = Bs / Ds; }
          if (Ds == T(0) && fl == LBX_FLUID_SPHERELIST) {
            T R2, B2;
            if (secbelt(b, i, j, k, R2, B2) != 0) { nR[x] = R2; nB[x] = B2; set[x] = 1; }
          } else {
            nR[x] = Rs; nB[x] = Bs; set[x] = 1;
          }
        }
    /* the reference writes in place; only fluid cells are read, so the
     * buffered write is the same */
    for (int64_t x = 0; x < ncell_pad; ++x)
      if (set[x]) { rho[0][x] = nR[x]; rho[1][x] = nB[x]; }
  }

  /* wall velocity of particle a at link lever r (lab frame) */
  void wall_vel(int b, int a, const P rt[3], const P ol[3], P v[3]) {
    P c[3];
    cross3(ol, rt, c);
    v[0] = ps(b, a, 3) + c[0];
    v[1] = ps(b, a, 4) + c[1];
    v[2] = ps(b, a, 5) + c[2];
  }

  /* links visited by the last step's n2p, one list per OpenMP thread */
  bool record_links = false;
  std::vector<std::vector<std::array<int64_t, 3>>> link_rec;
  void clear_links() {
#ifdef _OPENMP
    link_rec.assign(size_t(omp_get_max_threads()), {});
#else
    link_rec.assign(1, {});
#endif
  }
  std::vector<std::array<int64_t, 3>> links_sorted() const {
    std::vector<std::array<int64_t, 3>> all;
    for (const auto& v : link_rec) all.insert(all.end(), v.begin(), v.end());
    std::sort(all.begin(), all.end());
    return all;
  }

  /* node_to_particle_bounce_back_bc2, kernels_fluid_PART.CUF:1874-2113 */
  void n2p(int b, int a, int i, int j, int k) {
    P rv[3] = {0, 0, 0}, ol[3] = {0, 0, 0};
    if (lrotate) {
      P om[3] = {ps(b, a, 6), ps(b, a, 7), ps(b, a, 8)};
      to_lab(b, a, om, ol);
      lever(i, j, k, a, b, true, rv);
    }
    for (int it = 1; it <= 9; ++it) {
      int lo = 2 * it - 1, hi = 2 * it;
      int64_t xi = id(i + EX[lo], j + EY[lo], k + EZ[lo]);
      int64_t xo = id(i + EX[hi], j + EY[hi], k + EZ[hi]);
      for (int side = 0; side < 2; ++side) {
        int64_t xf = side ? xo : xi;        /* the fluid neighbour */
        int64_t xs = side ? xi : xo;        /* the opposite one, not fluid */
        int lf = side ? lo : hi;            /* direction of the population read at xf */
        int lr = side ? hi : lo;            /* direction towards xf */
        if (!(flags[b][xf] == LBX_FLUID_FLUID && flags[b][xs] != LBX_FLUID_FLUID)) continue;
        if (record_links) {
          /* the link this pair crosses: (sphere, surface cell, direction
           * towards the fluid end), the DEBUG_N2P record of the reference */
          const int64_t cell = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
#ifdef _OPENMP
          auto& out = link_rec[size_t(omp_get_thread_num())];
#else
          auto& out = link_rec[0];
#endif
          out.push_back({int64_t(a), cell, int64_t(lr)});
        }
        P v[3] = {ps(b, a, 3), ps(b, a, 4), ps(b, a, 5)};
        P rt[3] = {0, 0, 0};
        if (lrotate) {
          for (int d = 0; d < 3; ++d) rt[d] = rv[d] + P(0.5) * P(d == 0 ? EX[lr] : (d == 1 ? EY[lr] : EZ[lr]));
          wall_vel(b, a, rt, ol, v);
        }
        T ev = T(EX[lf]) * T(v[0]) + T(EY[lf]) * T(v[1]) + T(EZ[lf]) * T(v[2]);
        T f2pR = T(2) * f(0, b, lf, xf) - tb.p[lf] * buz * rho[0][xf] * ev;
        T f2pB = T(2) * f(1, b, lf, xf) - tb.p[lf] * buz * rho[1][xf] * ev;
        T f2p = f2pR + f2pB;
        T ft[3] = {f2p * T(EX[lf]), f2p * T(EY[lf]), f2p * T(EZ[lf])};
        double acc[3] = {double(ft[0]), double(ft[1]), double(ft[2])};
        add_acc(myf, a, acc);
        if (lrotate) {
          P t[3];
          cross3(rt, ft, t);
          double tt[3] = {double(t[0] * P(std::abs(EX[lf]))), double(t[1] * P(std::abs(EY[lf]))),
                          double(t[2] * P(std::abs(EZ[lf])))};
          add_acc(myt, a, tt);
        }
      }
    }
  }

  /* particle_to_node_bounce_back_bc2_phase1, kernels_fluid_PART.CUF:2153-2199 */
  void p2n_phase1(int b, int i, int j, int k) {
    int64_t x = id(i, j, k);
    for (int it = 1; it <= 9; ++it) {
      int lo = 2 * it - 1, hi = 2 * it;
      int64_t xi = id(i + EX[lo], j + EY[lo], k + EZ[lo]);
      int64_t xo = id(i + EX[hi], j + EY[hi], k + EZ[hi]);
      if (flags[b][xi] == LBX_FLUID_FLUID && flags[b][xo] != LBX_FLUID_FLUID)
        for (int c = 0; c < 2; ++c) f(c, b, lo, x) = f(c, b, hi, xi);
      if (flags[b][xi] != LBX_FLUID_FLUID && flags[b][xo] == LBX_FLUID_FLUID)
        for (int c = 0; c < 2; ++c) f(c, b, hi, x) = f(c, b, lo, xo);
    }
  }

  /* particle_to_node_bounce_back_bc2_phase2, kernels_fluid_PART.CUF:2201-2312 */
  void p2n_phase2(int b, int a, int i, int j, int k) {
    P rv[3] = {0, 0, 0}, ol[3] = {0, 0, 0};
    if (lrotate) {
      P om[3] = {ps(b, a, 6), ps(b, a, 7), ps(b, a, 8)};
      to_lab(b, a, om, ol);
      lever(i, j, k, a, b, true, rv);
    }
    int64_t x = id(i, j, k);
    for (int it = 1; it <= 9; ++it) {
      int lo = 2 * it - 1, hi = 2 * it;
      int64_t xi = id(i + EX[lo], j + EY[lo], k + EZ[lo]);
      int64_t xo = id(i + EX[hi], j + EY[hi], k + EZ[hi]);
      for (int side = 0; side < 2; ++side) {
        int64_t xf = side ? xo : xi;
        int64_t xs = side ? xi : xo;
        int lf = side ? lo : hi;
        int lr = side ? hi : lo;
        if (!(flags[b][xf] == LBX_FLUID_FLUID && flags[b][xs] != LBX_FLUID_FLUID)) continue;
        P v[3] = {ps(b, a, 3), ps(b, a, 4), ps(b, a, 5)};
        if (lrotate) {
          P rt[3];
          for (int d = 0; d < 3; ++d) rt[d] = rv[d] + P(0.5) * P(d == 0 ? EX[lr] : (d == 1 ? EY[lr] : EZ[lr]));
          wall_vel(b, a, rt, ol, v);
        }
        T ev = T(EX[lf]) * T(v[0]) + T(EY[lf]) * T(v[1]) + T(EZ[lf]) * T(v[2]);
        for (int c = 0; c < 2; ++c) f(c, b, lr, x) = f(c, b, lr, x) - tb.p[lf] * buz * rho[c][xf] * ev;
      }
    }
  }

  /* addHertzian (+ optional lubrication), kernels_fluid_PART.CUF:1385-1503 */
  void inter_forces(int b) {
    const P FIVE = 5, HALF = P(0.5), THREE = 3;
    const P hz_k = P(prm.hz_k), hz_rmin = P(prm.hz_rmin), hz_rcap = P(prm.hz_rcap);
    const P rsqcut = hz_rmin * hz_rmin;
    const P gmin = FIVE * HALF * hz_k * std::pow(hz_rmin - hz_rcap, THREE * HALF);
    const P rpar = P(2) * rdim;
    const P pi = P(3.141592653589793238462643383279502884);
    const P lubfactor = P(prm.lubric_k) * P(6) * pi * std::pow(rdim * rdim, P(2)) / (rpar * rpar);
    const P rparcut = rpar + P(prm.lubric_rmin);
    const P mxrsqcut = std::max(rparcut * rparcut, rsqcut);
    const P rparcap = rpar + P(prm.lubric_rcap);
    for (int ia = 0; ia < np; ++ia)
      for (int ja = ia + 1; ja < np; ++ja) {
        P xdf = ps(b, ja, 0) - ps(b, ia, 0), ydf = ps(b, ja, 1) - ps(b, ia, 1), zdf = ps(b, ja, 2) - ps(b, ia, 2);
        xdf = xdf - P(nx * nintp(xdf / P(nx)));
        ydf = ydf - P(ny * nintp(ydf / P(ny)));
        zdf = zdf - P(nz * nintp(zdf / P(nz)));
        P rsq = xdf * xdf + ydf * ydf + zdf * zdf;
        if (rsq > mxrsqcut) continue;
        P rrr = std::sqrt(rsq);
        if (rrr <= hz_rmin) {
          P ggg = (rrr <= hz_rcap) ? gmin : FIVE * HALF * hz_k * std::pow(hz_rmin - rrr, THREE * HALF);
          double ft[3] = {double(ggg * xdf / rrr), double(ggg * ydf / rrr), double(ggg * zdf / rrr)};
          for (int d = 0; d < 3; ++d) { myf2[3 * ia + d] -= ft[d]; myf2[3 * ja + d] += ft[d]; }
        }
        if (prm.lubrication && rrr <= rparcut) {
          P ux = xdf / rrr, uy = ydf / rrr, uz = zdf / rrr;
          if (rrr <= rparcap) rrr = rparcap;
          P dotuv = ux * (ps(b, ia, 3) - ps(b, ja, 3)) + uy * (ps(b, ia, 4) - ps(b, ja, 4)) + uz * (ps(b, ia, 5) - ps(b, ja, 5));
          P visc = 1;
          P c = visc * lubfactor * dotuv * (P(1) / (rrr - rpar) - P(1));
          double ft[3] = {double(c * ux), double(c * uy), double(c * uz)};
          /* the reference adds these to forceAtoms(1:3) without atomics; they
           * reach the integrator through the same total force */
          for (int d = 0; d < 3; ++d) { lub[3 * ia + d] -= ft[d]; lub[3 * ja + d] += ft[d]; }
        }
      }
  }
  std::vector<double> lub;

  /* time_step_force_particles: addForce_particle_bounce_back, nve_lf,
   * rot_midstep_impl_lf, kernels_fluid_PART.CUF:1098-1166,1266-1827 */
  void integrate(int b) {
    const int o = 1 - b;
    const P HALF = P(0.5), ONE = 1;
    const P rmass = P(prm.rmass), max_vel = P(prm.max_vel);
    const P mass = ONE / rmass;
    const P rotin = P(2) / P(5) * mass * rdim * rdim;
    const P cx = P(nx + 1) * HALF, cy = P(ny + 1) * HALF, cz = P(nz + 1) * HALF;
    for (int a = 0; a < np; ++a) {
      /* addForce_particle_bounce_back */
      for (int d = 0; d < 3; ++d) {
        fa(b, a, d) = P(myf2[3 * a + d]) + P(lub[3 * a + d]);
        fa(b, a, 3 + d) = P(myf[3 * a + d]);
        fa(b, a, d) = fa(b, a, d) + (fa(b, a, 3 + d) + fa(o, a, 3 + d)) * HALF;
      }
      if (lrotate)
        for (int d = 0; d < 3; ++d) {
          fa(b, a, 6 + d) = P(myt2[3 * a + d]);
          fa(b, a, 9 + d) = P(myt[3 * a + d]);
          fa(b, a, 6 + d) = fa(b, a, 6 + d) + (fa(b, a, 9 + d) + fa(o, a, 9 + d)) * HALF;
        }
      /* nve_lf */
      P xo[3] = {ps(b, a, 0), ps(b, a, 1), ps(b, a, 2)};
      P v[3] = {ps(b, a, 3), ps(b, a, 4), ps(b, a, 5)};
      P fr[3] = {fa(b, a, 0), fa(b, a, 1), fa(b, a, 2)};
      if (!prm.kinematic &&
          (std::abs(fr[0]) * rmass > P(0.5) || std::abs(fr[1]) * rmass > P(0.5) || std::abs(fr[2]) * rmass > P(0.5)))
        raise(LBX_DEV_BIG_FORCE, a);
      P bv[3];
      for (int d = 0; d < 3; ++d) bv[d] = prm.kinematic ? v[d] : v[d] + rmass * fr[d];
      P vm = std::sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
      if (!prm.kinematic && vm > max_vel) raise(LBX_DEV_EXTREME_VEL, a);
      P xn[3];
      for (int d = 0; d < 3; ++d) xn[d] = xo[d] + bv[d];
      const P cc[3] = {cx, cy, cz};
      const int nn[3] = {nx, ny, nz};
      for (int d = 0; d < 3; ++d) {
        P xs = xn[d] - cc[d];
        P aaa = ONE / P(nn[d]);
        xn[d] = xs - P(nn[d]) * P(nintp(aaa * xs)) + cc[d];
        if (xn[d] < P(0.5) || xn[d] > P(nn[d]) + P(0.5)) raise(LBX_DEV_POSITION, a);
      }
      if (lrotate) rot_midstep(b, a, rotin);
      for (int d = 0; d < 3; ++d) { ps(o, a, d) = xn[d]; ps(o, a, 3 + d) = bv[d]; }
      if (!lrotate)
        for (int c = 6; c < 13; ++c) ps(o, a, c) = ps(b, a, c);
      if (prm.kinematic) /* prescribed motion: centre moves with the set velocity, v / omega / q kept */
        for (int c = 3; c < 13; ++c) ps(o, a, c) = ps(b, a, c);
      if (prm.kinematic == 2) /* frozen geometry: centre stays, the wall still moves with v and omega */
        for (int c = 0; c < 3; ++c) ps(o, a, c) = ps(b, a, c);
      /* reset the accumulators to the external force / torque */
      for (int d = 0; d < 3; ++d) {
        fa(o, a, d) = P(prm.ext_force[d]);
        fa(o, a, 3 + d) = 0;
        myf[3 * a + d] = 0;
        myf2[3 * a + d] = double(prm.ext_force[d]);
        lub[3 * a + d] = 0;
        if (lrotate) {
          fa(o, a, 6 + d) = P(prm.ext_torque[d]);
          fa(o, a, 9 + d) = 0;
          myt[3 * a + d] = 0;
          myt2[3 * a + d] = double(prm.ext_torque[d]);
        }
      }
      oldpartVol[a] = partVol[a];
      partVol[a] = 0;
    }
  }

  /* rot_midstep_impl_lf, kernels_fluid_PART.CUF:1621-1827 */
  void rot_midstep(int b, int a, P rotin) {
    const int o = 1 - b;
    const P HALF = P(0.5), ONE = 1;
    const int mxquat = 20;
    const P sqquattol = P(1.0e-24);
    P oxx = ps(b, a, 6), oyy = ps(b, a, 7), ozz = ps(b, a, 8);
    P q0 = ps(b, a, 9), q1 = ps(b, a, 10), q2 = ps(b, a, 11), q3 = ps(b, a, 12);
    P tqx = fa(b, a, 6), tqy = fa(b, a, 7), tqz = fa(b, a, 8);
    P m[9];
    m[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
    m[1] = P(2) * (q1 * q2 - q0 * q3);
    m[2] = P(2) * (q1 * q3 + q0 * q2);
    m[3] = P(2) * (q1 * q2 + q0 * q3);
    m[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
    m[5] = P(2) * (q2 * q3 - q0 * q1);
    m[6] = P(2) * (q1 * q3 - q0 * q2);
    m[7] = P(2) * (q2 * q3 + q0 * q1);
    m[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
    P opx = oxx, opy = oyy, opz = ozz;
    const P rix = rotin, riy = rotin, riz = rotin;
    P trx = (tqx * m[0] + tqy * m[3] + tqz * m[6]) / rix + (riy - riz) * opy * opz / rix;
    P tr_y = (tqx * m[1] + tqy * m[4] + tqz * m[7]) / riy + (riz - rix) * opz * opx / riy;
    P trz = (tqx * m[2] + tqy * m[5] + tqz * m[8]) / riz + (rix - riy) * opx * opy / riz;
    P delx = trx, dely = tr_y, delz = trz;
    opx = oxx + delx * HALF;
    opy = oyy + dely * HALF;
    opz = ozz + delz * HALF;
    P dq0 = (-q1 * opx - q2 * opy - q3 * opz) * HALF;
    P dq1 = (q0 * opx - q3 * opy + q2 * opz) * HALF;
    P dq2 = (q3 * opx + q0 * opy - q1 * opz) * HALF;
    P dq3 = (-q2 * opx + q1 * opy + q0 * opz) * HALF;
    P qn0 = q0 + dq0 * HALF, qn1 = q1 + dq1 * HALF, qn2 = q2 + dq2 * HALF, qn3 = q3 + dq3 * HALF;
    P rnorm = ONE / std::sqrt(qn0 * qn0 + qn1 * qn1 + qn2 * qn2 + qn3 * qn3);
    qn0 *= rnorm; qn1 *= rnorm; qn2 *= rnorm; qn3 *= rnorm;
    oxx = oxx + delx;
    oyy = oyy + dely;
    ozz = ozz + delz;
    ps(o, a, 6) = oxx;
    ps(o, a, 7) = oyy;
    ps(o, a, 8) = ozz;
    opx = oxx; opy = oyy; opz = ozz;
    int itq = 0;
    P eps = P(1.0e9);
    while (itq < mxquat && eps > sqquattol) {
      itq += 1;
      dq0 = (-qn1 * opx - qn2 * opy - qn3 * opz) * HALF;
      dq1 = (qn0 * opx - qn3 * opy + qn2 * opz) * HALF;
      dq2 = (qn3 * opx + qn0 * opy - qn1 * opz) * HALF;
      dq3 = (-qn2 * opx + qn1 * opy + qn0 * opz) * HALF;
      P a0 = qn0 + dq0 * HALF, a1 = qn1 + dq1 * HALF, a2 = qn2 + dq2 * HALF, a3 = qn3 + dq3 * HALF;
      rnorm = ONE / std::sqrt(a0 * a0 + a1 * a1 + a2 * a2 + a3 * a3);
      a0 *= rnorm; a1 *= rnorm; a2 *= rnorm; a3 *= rnorm;
      eps = (a0 - qn0) * (a0 - qn0) + (a1 - qn1) * (a1 - qn1) + (a2 - qn2) * (a2 - qn2) + (a3 - qn3) * (a3 - qn3);
      qn0 = a0; qn1 = a1; qn2 = a2; qn3 = a3;
    }
    q0 = q0 + dq0; q1 = q1 + dq1; q2 = q2 + dq2; q3 = q3 + dq3;
    rnorm = ONE / std::sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    ps(o, a, 9) = q0 * rnorm;
    ps(o, a, 10) = q1 * rnorm;
    ps(o, a, 11) = q2 * rnorm;
    ps(o, a, 12) = q3 * rnorm;
  }

  void set_particles(int n, const double* x, const double* v, const double* om, const double* q) {
    np = n;
    lrotate = prm.lrotate != 0;
    rdim = P(prm.radius);
    buz = T(2) / tb.cssq; /* pref_bouzidi, dimensions_m.CUF:95 */
    for (int s2 = 0; s2 < 2; ++s2) {
      pos[s2].assign(13 * size_t(n), P(0));
      force[s2].assign(12 * size_t(n), P(0));
    }
    myf.assign(3 * size_t(n), 0); myf2 = myf; myt = myf; myt2 = myf; lub = myf;
    partVol.assign(n, 0); oldpartVol.assign(n, 0);
    owner.assign(ncell_pad, 0);
    for (int a = 0; a < n; ++a)
      for (int s2 = 0; s2 < 2; ++s2) {
        for (int d = 0; d < 3; ++d) {
          ps(s2, a, d) = P(x[3 * a + d]);
          ps(s2, a, 3 + d) = P(v[3 * a + d]);
          ps(s2, a, 6 + d) = om ? P(om[3 * a + d]) : P(0);
          fa(s2, a, d) = P(prm.ext_force[d]);
          if (lrotate) fa(s2, a, 6 + d) = P(prm.ext_torque[d]);
        }
        for (int c = 0; c < 4; ++c) ps(s2, a, 9 + c) = q ? P(q[4 * a + c]) : P(c == 0 ? 1 : 0);
      }
    nbx = nx / TX; nby = ny / TY; nbz = nz / TZ;
    tiles.assign(size_t(nbx) * nby * nbz, {});
    spherical_template();
    make_lists(flip);
    /* setupRho_Pops: init_isfluid_CG at step 0 + flag halo; partVol reset */
    init_isfluid(flip);
    last_flags = flip;
    std::fill(partVol.begin(), partVol.end(), 0);
  }

  void get_particles(double* x, double* v, double* om, double* q, double* fo, double* to) {
    int b = flip;
    for (int a = 0; a < np; ++a) {
      for (int d = 0; d < 3; ++d) {
        if (x) x[3 * a + d] = double(ps(b, a, d));
        if (v) v[3 * a + d] = double(ps(b, a, 3 + d));
        if (om) om[3 * a + d] = double(ps(b, a, 6 + d));
        /* the total force / torque the integrator used in the last step */
        if (fo) fo[3 * a + d] = double(fa(1 - b, a, d));
        if (to) to[3 * a + d] = double(fa(1 - b, a, 6 + d));
      }
      if (q)
        for (int c = 0; c < 4; ++c) q[4 * a + c] = double(ps(b, a, 9 + c));
    }
  }

  /* ---- one step with particles, main.CUF:130-241 --------------------------- */
  void do_step_particles() {
    step += 1;
    clear_links();
    const int b = flip;
    init_isfluid(b);
    for_cells_with_tile_atoms([&](int a, int i, int j, int k) {
      if (particle_moved(a)) del_fluid(b, a, i, j, k);
    });
    init_rho();
    for_cells_with_tile_atoms([&](int a, int i, int j, int k) {
      if (particle_moved(a)) make_fluid(b, a, i, j, k);
    });
    halo_rho();
    if (prm.wetting == LBX_WET_NEUTRAL) virtual_rho_neutral(b);
    else virtual_rho_janus(b);
    halo_rho();
    time_step_cg();
    /* partBB_CG: n2p for every tile atom within sphereMax of a spherelist node */
    for_cells_with_tile_atoms([&](int a, int i, int j, int k) {
      if (flags[b][id(i, j, k)] != LBX_FLUID_SPHERELIST) return;
      int di = getDelta(i, nintp(ps(b, a, 0)), nx), dj = getDelta(j, nintp(ps(b, a, 1)), ny),
          dk = getDelta(k, nintp(ps(b, a, 2)), nz);
      if (di * di + dj * dj + dk * dk < sphereMax) n2p(b, a, i, j, k);
    });
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          if (flags[b][id(i, j, k)] == LBX_FLUID_SPHERELIST) p2n_phase1(b, i, j, k);
    for_cells_with_tile_atoms([&](int a, int i, int j, int k) {
      if (flags[b][id(i, j, k)] != LBX_FLUID_SPHERELIST) return;
      int di = getDelta(i, nintp(ps(b, a, 0)), nx), dj = getDelta(j, nintp(ps(b, a, 1)), ny),
          dk = getDelta(k, nintp(ps(b, a, 2)), nz);
      if (di * di + dj * dj + dk * dk < sphereMax) p2n_phase2(b, a, i, j, k);
    });
    halo_pops(b);
    stream();
    inter_forces(b);
    integrate(b);
    make_lists(1 - b);
    last_flags = b;
    flip = 1 - flip;
  }

  /* ---- one step, main.CUF:125-308 (no particles) ----------------------------- */
  void do_step() {
    if (np > 0) { do_step_particles(); return; }
    step += 1;
    if (model != LBX_MODEL_BGK) {
      init_rho();
      time_step_cg();
    } else {
      time_step_bgk();
    }
    stream();
    last_flags = flip;
    flip = 1 - flip;
  }

  /* ---- moments2Fl, write_output.f90:975-1041 (on the current flip buffer) ---- */
  int last_flags = 0; /* flag slot of the last completed step (or of the setup) */
  void get_fields(double* oR, double* oB, double* vel, double* phase) {
    const int b = flip;
    const int bf = last_flags;
    const T ONE = 1, MINDENS = 0;
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          T pR[Q27], pB[Q27];
          for (int l = 0; l < q; ++l) { pR[l] = f(0, b, l, x); pB[l] = (ncomp == 2) ? f(1, b, l, x) : T(0); }
          T lr = pR[0], lb = pB[0];
          for (int l = 1; l < q; ++l) { lr = lr + pR[l]; lb = lb + pB[l]; }
          T rs = lr + lb;
          T inv = ONE / rs;
          /* moments2Fl (write_output.f90:975-1041) sums the R terms, then the
           * B terms, left to right; over all q directions (the reference's
           * routine lists only the first 19, also in its D3Q27 build) */
          T u = 0, v = 0, w = 0;
          for (int c = 0; c < 2; ++c) {
            const T* pp = c ? pB : pR;
            for (int l = 1; l < q; ++l) {
              if (EX[l]) u = EX[l] > 0 ? u + pp[l] : u - pp[l];
              if (EY[l]) v = EY[l] > 0 ? v + pp[l] : v - pp[l];
              if (EZ[l]) w = EZ[l] > 0 ? w + pp[l] : w - pp[l];
            }
          }
          u = inv * u;
          v = inv * v;
          w = inv * w;
          bool ok = flags[bf][x] == LBX_FLUID_FLUID && rs > MINDENS;
          if (oR) oR[h] = ok ? double(lr) : 0.0;
          if (oB) oB[h] = ok ? double(lb) : 0.0;
          if (vel) {
            vel[3 * h + 0] = ok ? double(u) : 0.0;
            vel[3 * h + 1] = ok ? double(v) : 0.0;
            vel[3 * h + 2] = ok ? double(w) : 0.0;
          }
          if (phase) phase[h] = ok ? double((lr - lb) / (lr + lb)) : 0.0;
        }
  }

  void get_pops(double* pR, double* pB) {
    const int b = flip;
    int ncomp = (model != LBX_MODEL_BGK) ? 2 : 1;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          for (int l = 0; l < q; ++l) {
            if (pR) pR[h + n * l] = double(f(0, b, l, x));
            if (pB) pB[h + n * l] = (ncomp == 2) ? double(f(1, b, l, x)) : 0.0;
          }
        }
  }

  void get_flags(int8_t* out) {
    const int b = last_flags;
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i)
          out[(i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1))] = flags[b][id(i, j, k)];
  }
};

struct Handle {
  int mode;
  void* o;
};

template <typename F>
int dispatch(void* h, F&& fn) {
  if (!h) return LBX_ERR_ARG;
  Handle* H = static_cast<Handle*>(h);
  switch (H->mode) {
    case 0: return fn(*static_cast<Oracle<float, float>*>(H->o));
    case 1: return fn(*static_cast<Oracle<float, double>*>(H->o));
    case 2: return fn(*static_cast<Oracle<double, double>*>(H->o));
  }
  return LBX_ERR_ARG;
}

}  // namespace

extern "C" {

/* mode: 0 = reference precision (FP32 fluid, FP32 particles), 1 = FP32 fluid
 * with FP64 particle state, 2 = FP64 everything */
void* orc_create(const lbx_params* p, int mode) {
  if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return nullptr;
  Handle* H = new Handle{mode, nullptr};
  switch (mode) {
    case 0: H->o = new Oracle<float, float>(*p); break;
    case 1: H->o = new Oracle<float, double>(*p); break;
    case 2: H->o = new Oracle<double, double>(*p); break;
    default: delete H; return nullptr;
  }
  return H;
}

void orc_destroy(void* h) {
  if (!h) return;
  Handle* H = static_cast<Handle*>(h);
  switch (H->mode) {
    case 0: delete static_cast<Oracle<float, float>*>(H->o); break;
    case 1: delete static_cast<Oracle<float, double>*>(H->o); break;
    case 2: delete static_cast<Oracle<double, double>*>(H->o); break;
  }
  delete H;
}

int orc_set_fields(void* h, const float* rR, const float* rB, float vx, float vy, float vz) {
  return dispatch(h, [&](auto& o) { o.set_fields(rR, rB, vx, vy, vz); return 0; });
}
int orc_set_pops(void* h, const float* pR, const float* pB) {
  return dispatch(h, [&](auto& o) { o.set_pops(pR, pB); return 0; });
}
int orc_step(void* h, int n) {
  return dispatch(h, [&](auto& o) {
    for (int s = 0; s < n; ++s) o.do_step();
    return o.err_code;
  });
}
int orc_get_fields(void* h, double* rR, double* rB, double* vel, double* phase) {
  return dispatch(h, [&](auto& o) { o.get_fields(rR, rB, vel, phase); return 0; });
}
int orc_get_pops(void* h, double* pR, double* pB) {
  return dispatch(h, [&](auto& o) { o.get_pops(pR, pB); return 0; });
}
int orc_get_flags(void* h, int8_t* out) {
  return dispatch(h, [&](auto& o) { o.get_flags(out); return 0; });
}
int orc_status(void* h, int* code, int* step, int64_t* where) {
  return dispatch(h, [&](auto& o) {
    if (code) *code = o.err_code;
    if (step) *step = o.err_step;
    if (where) *where = o.err_where;
    o.err_code = 0;
    return 0;
  });
}
int orc_set_particles(void* h, int n, const double* x, const double* v, const double* om, const double* q) {
  return dispatch(h, [&](auto& o) {
    if (o.model == LBX_MODEL_BGK || n < 1) return int(LBX_ERR_ARG);
    if (o.nx % 8 || o.ny % 4 || o.nz % 4) return int(LBX_ERR_ARG); /* reference tile 8x4x4 */
    o.set_particles(n, x, v, om, q);
    return o.err_code;
  });
}
int orc_get_particles(void* h, double* x, double* v, double* om, double* q, double* fo, double* to) {
  return dispatch(h, [&](auto& o) { o.get_particles(x, v, om, q, fo, to); return 0; });
}
/* accumulators of the current step: myf (bounce-back), myf2 (fill/drain +
 * pair + external), myt, myt2, each 3*np */
int orc_get_accumulators(void* h, double* f_bb, double* f_other, double* t_bb, double* t_other) {
  return dispatch(h, [&](auto& o) {
    for (size_t i = 0; i < o.myf.size(); ++i) {
      if (f_bb) f_bb[i] = o.myf[i];
      if (f_other) f_other[i] = o.myf2[i];
      if (t_bb) t_bb[i] = o.myt[i];
      if (t_other) t_other[i] = o.myt2[i];
    }
    return 0;
  });
}
int orc_get_rho(void* h, double* rR, double* rB) {
  return dispatch(h, [&](auto& o) {
    for (int k = 1; k <= o.nz; ++k)
      for (int j = 1; j <= o.ny; ++j)
        for (int i = 1; i <= o.nx; ++i) {
          int64_t x = o.id(i, j, k);
          int64_t hh = (i - 1) + int64_t(o.nx) * ((j - 1) + int64_t(o.ny) * (k - 1));
          if (rR) rR[hh] = double(o.rho[0][x]);
          if (rB) rB[hh] = double(o.rho[1][x]);
        }
    return 0;
  });
}
int orc_template(void* h, int* rmax, int8_t* out) {
  return dispatch(h, [&](auto& o) {
    if (rmax) *rmax = o.rmax;
    if (out) for (size_t i = 0; i < o.issub.size(); ++i) out[i] = o.issub[i];
    return 0;
  });
}
/* the reference defaults of lbx_params (dimensions_m.CUF:50-99): the
 * compile-time parameters of the reference, restated for the oracle's own
 * callers */
void orc_default_params(lbx_params* p, int32_t nx, int32_t ny, int32_t nz) {
  std::memset(p, 0, sizeof(*p));
  p->nx = nx; p->ny = ny; p->nz = nz;
  p->model = LBX_MODEL_CG;
  p->storage = LBX_STORE_F32;
  p->wetting = LBX_WET_JANUS;
  p->tau = 1.0f;
  p->tauR = 1.0f; p->tauB = 1.0f;       /* dimensions_m.CUF:98-99 */
  p->sigma = 0.1f; p->beta = 0.999f;    /* dimensions_m.CUF:50 */
  p->rho0R = 0.5f; p->rho0B = 0.5f;
  p->radius = 5.5f;                     /* dimensions_m.CUF:59 */
  p->rmass = 1.0f / 1500.0f;            /* dimensions_m.CUF:60 */
  p->hz_k = 10.0f; p->hz_rmin = 10.5f; p->hz_rcap = 9.0f;               /* :77-80 */
  p->lubric_k = 10.0f; p->lubric_rmin = 10.0f; p->lubric_rcap = 9.0f;  /* :81-84 */
  p->closure_gap_min = 0.05f; p->closure_gap_max = 1.5f; p->closure_vmax = 1.0e-3f;
  p->exact_tiles = 1;
  p->densR = 1.0f; p->densB = 1.0f;     /* noDIFFDENS, main.CUF:1065-1066 */
}

/* the boundary links of the last step's bounce-back (record_links on), as
 * (sphere, cell, direction) sorted; *n = total, at most cap written */
int orc_record_links(void* h, int on) {
  return dispatch(h, [&](auto& o) { o.record_links = on != 0; if (on) o.clear_links(); return 0; });
}
int orc_get_links(void* h, int32_t* cell, int8_t* dir, int32_t* sph, int64_t cap, int64_t* n) {
  return dispatch(h, [&](auto& o) {
    auto all = o.links_sorted();
    *n = int64_t(all.size());
    for (size_t i = 0; i < all.size() && int64_t(i) < cap; ++i) {
      sph[i] = int32_t(all[i][0]);
      cell[i] = int32_t(all[i][1]);
      dir[i] = int8_t(all[i][2]);
    }
    return 0;
  });
}
int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
