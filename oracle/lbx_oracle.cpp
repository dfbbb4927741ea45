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
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/lbx.h"

namespace {

constexpr int Q = 19;
constexpr int Q27 = 27;

/* ---- lattice tables, dimensions_m.CUF:201-300 (D3Q19, noD3Q27) ------------- */
const int EX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
const int EY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1};
const int EZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
/* D3Q27 neighbour set used by HIGHGRAD and the belts, dimensions_m.CUF:275-281 */
const int EX27[Q27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
const int EY27[Q27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1};
const int EZ27[Q27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};

template <typename T>
struct Tables {
  T p[Q], b_l[Q], rec_fact[Q], a27[Q27], p27[Q27];
  T cssq;
  Tables() {
    /* all arithmetic in T, in the order the Fortran parameter expressions use */
    const T ONE = 1, TWO = 2, THREE = 3, SIX = 6, TWELVE = 12, TWENTYFOUR = 24;
    cssq = T(1.0) / T(3.0);                                   /* dimensions_m.CUF:94 */
    const T p0 = T(1.0) / T(3.0), p1 = T(1.0) / T(18.0), p2 = T(1.0) / T(36.0); /* :208-210 */
    for (int l = 0; l < Q; ++l) p[l] = (l == 0) ? p0 : (l <= 6 ? p1 : p2);
    const T b_xi = T(0.5);                                    /* Leclaire, :222 */
    const T b0 = -(TWO + TWO * b_xi) / (THREE * b_xi + TWELVE);
    const T b1 = (b_xi) / (SIX * b_xi + TWENTYFOUR);
    const T b2 = ONE / (SIX * b_xi + TWENTYFOUR);
    for (int l = 0; l < Q; ++l) b_l[l] = (l == 0) ? b0 : (l <= 6 ? b1 : b2);
    for (int l = 0; l < Q; ++l) /* SetConstants, main.CUF:1098 */
      rec_fact[l] = std::sqrt(T(EX[l] * EX[l] + EY[l] * EY[l] + EZ[l] * EZ[l]));
    const T q0 = (TWO / THREE) * (TWO / THREE) * (TWO / THREE);   /* :283-286 */
    const T q1 = (TWO / THREE) * (TWO / THREE) * (ONE / SIX);
    const T q2 = (ONE / SIX) * (ONE / SIX) * (TWO / THREE);
    const T q3 = (ONE / SIX) * (ONE / SIX) * (ONE / SIX);
    for (int l = 0; l < Q27; ++l) {
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

  Oracle(const lbx_params& p) : prm(p) {
    nx = p.nx; ny = p.ny; nz = p.nz;
    sx = nx + 2; sy = ny + 2; sz = nz + 2;
    ncell_pad = int64_t(sx) * sy * sz;
    model = p.model;
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
    for (int c = 0; c < ncomp; ++c)
      for (int b = 0; b < 2; ++b) pops[c][b].assign(size_t(Q) * ncell_pad, T(0));
    for (int c = 0; c < 2; ++c) rho[c].assign(ncell_pad, T(0));
    for (int b = 0; b < 2; ++b) flags[b].assign(ncell_pad, int8_t(LBX_FLUID_FLUID));
    const T HALF = T(0.5);
    viscR = tb.cssq * (T(p.tauR) - HALF); /* main.CUF:1069-1071 */
    viscB = tb.cssq * (T(p.tauB) - HALF);
    omega_bgk = T(1) / T(p.tau);
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
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
    for_halo([&](int64_t h, int64_t s) {
      for (int c = 0; c < ncomp; ++c)
        for (int l = 1; l < Q; ++l) f(c, b, l, h) = f(c, b, l, s);
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
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
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
          for (int l = 0; l < Q; ++l) {
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
  }

  void set_pops(const float* pR, const float* pB) {
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
    flip = 0;
    step = 0;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          int64_t x = id(i, j, k);
          for (int l = 0; l < Q; ++l) {
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
              for (int l = 1; l < Q; ++l) r = r + f(c, b, l, x); /* fixed order 0..18 */
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
  static inline T mom_x(const T* q, T inv) { return inv * (q[1] - q[2] + q[7] - q[8] - q[9] + q[10] + q[11] - q[12] - q[13] + q[14]); }
  static inline T mom_y(const T* q, T inv) { return inv * (q[3] - q[4] + q[7] - q[8] + q[9] - q[10] + q[15] - q[16] - q[17] + q[18]); }
  static inline T mom_z(const T* q, T inv) { return inv * (q[5] - q[6] + q[11] - q[12] + q[13] - q[14] + q[15] - q[16] + q[17] - q[18]); }

  /* ---- time_step_CG, kernels_fluid_CG.CUF:531-848 (noDIFFDENS, HIGHGRAD) ------ */
  void time_step_cg() {
    const T ONE = 1, HALF = T(0.5), ZERO = 0, NINE = 9, FOUR = 4;
    const T mylimit = T(1.e-20);
    const T sigma = T(prm.sigma), beta = T(prm.beta);
    const T densR = 1, densB = 1; /* noDIFFDENS: SetConstants main.CUF:1062-1067 */
    const int b = flip;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          if (flags[b][x] != LBX_FLUID_FLUID) continue;
          T tR[Q], tB[Q], fd[Q];
          for (int l = 0; l < Q; ++l) { tR[l] = f(0, b, l, x); tB[l] = f(1, b, l, x); }
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
          for (int l = 1; l < Q27; ++l) { /* HIGHGRAD, :720-741 */
            int64_t y = id(i + EX27[l], j + EY27[l], k + EZ27[l]);
            T rs = rho[0][y], bs = rho[1][y];
            T ps = (rs / densR - bs / densB) / (rs / densR + bs / densB);
            psix = psix + tb.a27[l] * T(EX27[l]) * ps;
            psiy = psiy + tb.a27[l] * T(EY27[l]) * ps;
            psiz = psiz + tb.a27[l] * T(EZ27[l]) * ps;
          }
          for (int l = 0; l < Q; ++l) tR[l] = tR[l] * oneminusomega + equil(tb, rhoR, u, v, w, l) * omega;
          for (int l = 0; l < Q; ++l) tB[l] = tB[l] * oneminusomega + equil(tb, rhoB, u, v, w, l) * omega;
          T psinorm_sq = psix * psix + psiy * psiy + psiz * psiz;
          if (psinorm_sq > mylimit) { /* perturbation + recolouring, :803-837 */
            T psinorm = std::sqrt(psinorm_sq);
            T acoeff = NINE / FOUR * omega * sigma;
            for (int l = 0; l < Q; ++l) {
              T edp = T(EX[l]) * psix + T(EY[l]) * psiy + T(EZ[l]) * psiz;
              T temp = psinorm * (tb.p[l] * (edp * edp) / psinorm_sq - tb.b_l[l]);
              fd[l] = tR[l] + tB[l] + acoeff * temp;
            }
            for (int l = 0; l < Q; ++l) {
              T feq = equil(tb, rhoR, ZERO, ZERO, ZERO, l) + equil(tb, rhoB, ZERO, ZERO, ZERO, l);
              T edp = T(EX[l]) * psix + T(EY[l]) * psiy + T(EZ[l]) * psiz;
              T temp1 = tb.rec_fact[l] * psinorm;
              T cosphi = (temp1 <= mylimit) ? ZERO : edp / temp1;
              T temp = beta * rhoR * rhoB * cosphi / (rhosum * rhosum);
              f(0, b, l, x) = fd[l] * rhoR / rhosum + temp * feq;
              f(1, b, l, x) = fd[l] * rhoB / rhosum - temp * feq;
            }
          } else {
            for (int l = 0; l < Q; ++l) { f(0, b, l, x) = tR[l]; f(1, b, l, x) = tB[l]; }
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
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
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
            for (int l = 1; l < Q; ++l) f(c, o, l, id(i + EX[l], j + EY[l], k + EZ[l])) = f(c, b, l, x);
        }
    /* halo cells push into the interior (stream_CG_x, _y, _z) */
    auto halo_push = [&](int i, int j, int k) {
      int64_t x = id(i, j, k);
      if (flags[b][x] == LBX_FLUID_SPHEREDEAD) return;
      for (int l = 1; l < Q; ++l) {
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

  /* ---- one step, main.CUF:125-308 (no particles) ----------------------------- */
  void do_step() {
    step += 1;
    if (model == LBX_MODEL_CG) {
      init_rho();
      time_step_cg();
    } else {
      time_step_bgk();
    }
    stream();
    flip = 1 - flip;
  }

  /* ---- moments2Fl, write_output.f90:975-1041 (on the current flip buffer) ---- */
  void get_fields(double* oR, double* oB, double* vel, double* phase) {
    const int b = flip;
    const T ONE = 1, MINDENS = 0;
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          T pR[Q], pB[Q];
          for (int l = 0; l < Q; ++l) { pR[l] = f(0, b, l, x); pB[l] = (ncomp == 2) ? f(1, b, l, x) : T(0); }
          T lr = pR[0], lb = pB[0];
          for (int l = 1; l < Q; ++l) { lr = lr + pR[l]; lb = lb + pB[l]; }
          T rs = lr + lb;
          T inv = ONE / rs;
          T u = inv * (pR[1] - pR[2] + pR[7] - pR[8] - pR[9] + pR[10] + pR[11] - pR[12] - pR[13] + pR[14] +
                       pB[1] - pB[2] + pB[7] - pB[8] - pB[9] + pB[10] + pB[11] - pB[12] - pB[13] + pB[14]);
          T v = inv * (pR[3] - pR[4] + pR[7] - pR[8] + pR[9] - pR[10] + pR[15] - pR[16] - pR[17] + pR[18] +
                       pB[3] - pB[4] + pB[7] - pB[8] + pB[9] - pB[10] + pB[15] - pB[16] - pB[17] + pB[18]);
          T w = inv * (pR[5] - pR[6] + pR[11] - pR[12] + pR[13] - pR[14] + pR[15] - pR[16] + pR[17] - pR[18] +
                       pB[5] - pB[6] + pB[11] - pB[12] + pB[13] - pB[14] + pB[15] - pB[16] + pB[17] - pB[18]);
          bool ok = flags[b][x] == LBX_FLUID_FLUID && rs > MINDENS;
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
    int ncomp = (model == LBX_MODEL_CG) ? 2 : 1;
    int64_t n = int64_t(nx) * ny * nz;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          int64_t x = id(i, j, k);
          int64_t h = (i - 1) + int64_t(nx) * ((j - 1) + int64_t(ny) * (k - 1));
          for (int l = 0; l < Q; ++l) {
            if (pR) pR[h + n * l] = double(f(0, b, l, x));
            if (pB) pB[h + n * l] = (ncomp == 2) ? double(f(1, b, l, x)) : 0.0;
          }
        }
  }

  void get_flags(int8_t* out) {
    const int b = 1 - flip; /* flags of the last step taken */
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
int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
