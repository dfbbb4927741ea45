// lbx_particles.cu — rigid spheres of the LBcuda hot path on sm_100a.
//
// Reference behaviour restated (kernels_fluid_PART.CUF unless noted):
//   spherical_template (main.CUF:1990-2130)        -> host, uploaded once
//   makeListAtomsGPU (2331-2451)                    -> k_bins (+ the tile-list
//                                                      coverage predicate)
//   init_isfluid_CG + setmyfluid (85-117,230-264)   -> k_stamp, k_stamp_flags
//   del_fluid_CG / del_fluid (120-149,383-561)      -> k_drain
//   init_rhoR_CG / init_rhoB_CG (CG.CUF:398-509)    -> k_rho_p
//   make_fluid_CG / make_fluid + belts (152-180,563-913) -> k_fill
//   compute_virtual_rho / compute_densities_wall (267-352) -> k_virtual
//   time_step_CG (CG.CUF:531-848)                   -> k_collide_p
//   partBB_CG, partBB_CG_p2n, partBB_CG_p2n2 (916-1040,1874-2312) -> k_bb
//   inter_force_particles / addHertzian (1052-1068,1385-1503) -> k_pairs
//   time_step_force_particles, addForce_particle_bounce_back, nve_lf,
//   rot_midstep_impl_lf (1098-1166,1266-1827)       -> k_integrate
//
// B200 design: particle state, orientation and every force/torque sum are
// FP64.  Each per-particle kernel is one CTA per sphere that walks a list of
// cell offsets around the sphere's centre (the template's solid cells, or
// the cells within its reach), so the momentum exchanged at the
// surface links is reduced inside the CTA in a fixed order and written once
// per step (no global atomics, bit-reproducible), instead of one FP64 atomic
// per link.  Per-cell work that must happen once per cell (the bounce-back
// copy and moving-wall correction) is done by the sphere that owns the cell.
// The fluid kernels of a particle step read the flags of the previous step
// for the pull (a spheredead source keeps the stale population, as the push
// of stream*_CG leaves it) and of the current step for the collision.
#include "lbx_device.cuh"
#include "lbx_closure.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace lbx {

constexpr int PS = 13;   // pos record: x[3] v[3] omega_body[3] q[4]
constexpr int FS = 12;   // force record: F[3] F_bb[3] T[3] T_bb[3]
constexpr int AS = 15;   // accumulators: f_bb[3] t_bb[3] f_other[3] t_other[3] f_lub[3]
constexpr int TILEX = 8, TILEY = 4, TILEZ = 4;  // reference tile (defines.h:14-22)
constexpr int BINW = 8;                          // cell bins of the particle lists
constexpr int BIN_CAP = 64;
constexpr int NBCAP = 32;                        // close neighbours per sphere (closure)

struct ParticleState {
  int np = 0;
  int rmax = 0, sphereMax = 0, tw = 0;
  double rdim = 0;
  int lrotate = 0;
  double* pos[2] = {nullptr, nullptr};
  double* frc[2] = {nullptr, nullptr};
  double* acc = nullptr;
  int8_t* tmpl = nullptr;
  int* offs = nullptr;        // packed template offsets (pack_off): solid cells, then the bounce-back list
  int n_surf = 0, n_solid = 0, n_bb = 0, n_shell = 0, shell_r2 = 0;
  int* owner = nullptr;       // lowest index of the spheres whose template holds the cell, -1 if none
  int* bin_cnt = nullptr;
  int* bin_list = nullptr;
  int nbx = 0, nby = 0, nbz = 0;
  int pcur = 0;
  int flags_last = 0;
  int active = 0;
  // learned closure
  float* wclosure = nullptr;  // LBX_CLOSURE_NWEIGHTS
  int closure_ready = 0;
  int* nbr = nullptr;         // np x NBCAP
  int* nbr_cnt = nullptr;
  float* corr = nullptr;      // np x NBCAP x 12
  int8_t* crowd = nullptr;    // per sphere: another sphere's template can reach into its bounce-back reach
  // second stream of the step's post stage: the pair forces and the
  // clearing of the previous flags run beside the bounce-back
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_flags = nullptr, ev_owner = nullptr;
  // the owners of the last stamping are already cleared (the end of the
  // step did it beside the integrator): the next flag stage skips that
  int owner_clear = 0;
};

struct PDev {  // by-value kernel argument
  int np, rmax, sphereMax, tw, lrotate;
  double rdim, rmass, max_vel;
  const int8_t* tmpl;
  const int* offs;     // [0, n_surf) surface offsets, [n_surf, n_solid) dead + centre
  const int* offs_bb;  // surface offsets, then the other offsets with d^2 < sphereMax
  const int* offs_shell;  // offsets with d^2 <= shell_r2 (the density shell)
  int n_surf, n_solid, n_bb, n_shell, shell_r2;
  int* owner;
  int* bin_cnt;
  int* bin_list;
  int nbx, nby, nbz;
  double ext_f[3], ext_t[3];
  double hz_k, hz_rmin, hz_rcap;
  int lub;
  double lub_k, lub_rmin, lub_rcap;
  int kinematic;
  int closure;
  float cl_gmin, cl_gmax, cl_vmax;
  int exact_tiles;
  int8_t* crowd;  // k_crowd's vote per sphere, read by k_bb
};

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int nint_d(double x) { return int(round(x)); }  // Fortran NINT
// NINT of a coordinate used to index the lattice: a non-finite or far
// out-of-box value (the integrator has already raised LBX_DEV_POSITION for it)
// maps to cell 1 so that no index leaves the arrays
__device__ __forceinline__ int nint_idx(double x, int n) {
  return (x > -double(n) && x < 2.0 * double(n)) ? int(round(x)) : 1;
}

// getDeltai/j/k (kernels_fluid_PART.CUF:182-228)
__device__ __forceinline__ int get_delta(int i, int c, int n, double rdim) {
  int d = i - c;
  if (double(c) - rdim < 1.0 || double(c) + rdim > double(n)) {
    if (double(c) + rdim > double(n) && double(i) < rdim) d = i - c + n;
    else if (double(c) - rdim < 1.0 && double(i) > double(n) - rdim) d = i - c - n;
  }
  return d;
}

// 1-based lattice coordinate (reference convention) of c0 + d, periodic
__device__ __forceinline__ int wrap1(int v, int n) {
  v = (v - 1) % n;
  if (v < 0) v += n;
  return v + 1;
}

__device__ __forceinline__ int cell0(const Geom& g, int i1, int j1, int k1) {  // 1-based -> linear
  return (i1 - 1) + g.nx * ((j1 - 1) + g.ny * (k1 - 1));
}

// template offset (dx, dy, dz) and template value packed in one word
__host__ __device__ __forceinline__ int pack_off(int dx, int dy, int dz, int v) {
  return (dx + 64) | ((dy + 64) << 8) | ((dz + 64) << 16) | (v << 24);
}
__device__ __forceinline__ void unpack_off(int w, int& dx, int& dy, int& dz, int& v) {
  dx = (w & 255) - 64;
  dy = ((w >> 8) & 255) - 64;
  dz = ((w >> 16) & 255) - 64;
  v = (w >> 24) & 255;
}

// cell of sphere offset d around centre c, when d is the offset getDelta
// assigns to that cell (the reference visits each cell under that offset only)
__device__ __forceinline__ bool offset_cell(const PDev& P, const Geom& g, const int c[3], int dx, int dy, int dz,
                                            int& i1, int& j1, int& k1) {
  i1 = wrap1(c[0] + dx, g.nx);
  j1 = wrap1(c[1] + dy, g.ny);
  k1 = wrap1(c[2] + dz, g.nz);
  return get_delta(i1, c[0], g.nx, P.rdim) == dx && get_delta(j1, c[1], g.ny, P.rdim) == dy &&
         get_delta(k1, c[2], g.nz, P.rdim) == dz;
}

// whether the (2 rmax + 1)^3 box around centre c lies inside the lattice:
// then no offset of the template lists (|d| <= rmax, and rdim <= rmax)
// wraps, getDelta is the plain difference, and offset_cell is the sum c + d
// for every offset
__device__ __forceinline__ bool box_inside(const PDev& P, const Geom& g, const int c[3]) {
  return c[0] - P.rmax >= 1 && c[0] + P.rmax <= g.nx && c[1] - P.rmax >= 1 && c[1] + P.rmax <= g.ny &&
         c[2] - P.rmax >= 1 && c[2] + P.rmax <= g.nz;
}
__device__ __forceinline__ bool offset_cell_in(const PDev& P, const Geom& g, bool inside, const int c[3], int dx,
                                               int dy, int dz, int& i1, int& j1, int& k1) {
  if (inside) {
    i1 = c[0] + dx;
    j1 = c[1] + dy;
    k1 = c[2] + dz;
    return true;
  }
  return offset_cell(P, g, c, dx, dy, dz, i1, j1, k1);
}

// Tile-list coverage of makeListAtomsGPU: the reference's 8x4x4 tiles
// (1-based indices) that hold particle position x in the list of the current
// step, as two ranges [lo0, hi0] and [lo1, hi1] per axis (R[4 d + 0..3]).
__device__ void tile_ranges(const double x[3], const int n[3], double rdim, int R[12]) {
  const int td[3] = {TILEX, TILEY, TILEZ};
  for (int d = 0; d < 3; ++d) {
    int ci = int(ceil(x[d]));
    int b0 = int(x[d] - rdim), b1 = int(x[d] + rdim), b2, b3;  // real -> integer truncation
    if (b0 < 1) {
      b0 = 1; b1 = int(double(ci) + rdim); b2 = int(double(ci) - rdim + double(n[d])); b3 = n[d];
    } else if (b1 > n[d]) {
      b0 = 1; b1 = int(double(ci) + rdim - double(n[d])); b2 = int(double(ci) - rdim); b3 = n[d];
    } else {
      b2 = td[d]; b3 = -td[d];
    }
    R[4 * d + 0] = (b0 - 1) / td[d] + 1;
    R[4 * d + 1] = (b1 - 1) / td[d] + 1;
    R[4 * d + 2] = (b2 - 1) / td[d] + 1;
    R[4 * d + 3] = (b3 - 1) / td[d] + 1;
  }
}
__device__ __forceinline__ bool in_tile_ranges(const int* R, int ti, int tj, int tk) {
  const int t[3] = {ti, tj, tk};
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    ok = ok && ((t[d] >= R[4 * d] && t[d] <= R[4 * d + 1]) || (t[d] >= R[4 * d + 2] && t[d] <= R[4 * d + 3]));
  return ok;
}
// whether the tile (ti, tj, tk) holds particle position x
__device__ bool tile_covered(const double x[3], const int n[3], double rdim, int ti, int tj, int tk) {
  int R[12];
  tile_ranges(x, n, rdim, R);
  return in_tile_ranges(R, ti, tj, tk);
}

// q (0,v) q*  (qtrimult, kernels_fluid_PART.CUF:1830-1871)
__device__ __forceinline__ void qmult(const double a[4], const double b[4], double o[4]) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  double c0 = a[2] * b[3] - a[3] * b[2], c1 = a[3] * b[1] - a[1] * b[3], c2 = a[1] * b[2] - a[2] * b[1];
  o[1] = a[0] * b[1] + b[0] * a[1] + c0;
  o[2] = a[0] * b[2] + b[0] * a[2] + c1;
  o[3] = a[0] * b[3] + b[0] * a[3] + c2;
}
__device__ __forceinline__ void to_lab(const double* P, const double v[3], double out[3]) {
  double q[4] = {P[9], P[10], P[11], P[12]};
  double qc[4] = {q[0], -q[1], -q[2], -q[3]};
  double qv[4] = {0.0, v[0], v[1], v[2]};
  double t[4], o[4];
  qmult(qv, qc, t);
  qmult(q, t, o);
  out[0] = o[1]; out[1] = o[2]; out[2] = o[3];
}

// min-image lever from the particle centre to cell (i,j,k), scaled to rdim
__device__ __forceinline__ void lever(const Geom& g, const double* P, int i, int j, int k, bool image, double rdim,
                                      double r[3]) {
  r[0] = double(i) - P[0];
  r[1] = double(j) - P[1];
  r[2] = double(k) - P[2];
  if (image) {
    r[0] = r[0] - double(g.nx) * double(nint_d((1.0 / g.nx) * r[0]));
    r[1] = r[1] - double(g.ny) * double(nint_d((1.0 / g.ny) * r[1]));
    r[2] = r[2] - double(g.nz) * double(nint_d((1.0 / g.nz) * r[2]));
  }
  double m = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  for (int d = 0; d < 3; ++d) r[d] = rdim / m * r[d];
}

__device__ __forceinline__ void cross(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// both components of a direction and cell (adjacent, aligned to their pair)
// in one load / store
__device__ __forceinline__ void ld_two(const __half* p, __half& a, __half& b) {
  const __half2 v = __ldg(reinterpret_cast<const __half2*>(p));
  a = __low2half(v);
  b = __high2half(v);
}
__device__ __forceinline__ void ld_two(const __nv_bfloat16* p, __nv_bfloat16& a, __nv_bfloat16& b) {
  const __nv_bfloat162 v = __ldg(reinterpret_cast<const __nv_bfloat162*>(p));
  a = __low2bfloat16(v);
  b = __high2bfloat16(v);
}
__device__ __forceinline__ void ld_two(const float* p, float& a, float& b) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ld_two(const double* p, double& a, double& b) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void st_two(__half* p, __half a, __half b) {
  *reinterpret_cast<__half2*>(p) = __halves2half2(a, b);
}
__device__ __forceinline__ void st_two(__nv_bfloat16* p, __nv_bfloat16 a, __nv_bfloat16 b) {
  *reinterpret_cast<__nv_bfloat162*>(p) = __halves2bfloat162(a, b);
}
__device__ __forceinline__ void st_two(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
__device__ __forceinline__ void st_two(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

// fixed-order CTA reduction of NV doubles (blockDim.x == 256)
template <int NV>
__device__ void block_sum(double v[NV], double* out /* NV, added */) {
  __shared__ double red[8][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  if (lane == 0)
    for (int i = 0; i < NV; ++i) red[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < NV; ++i) {
      double s = 0;
      for (int w = 0; w < 8; ++w) s += red[w][i];
      out[i] += s;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// one warp per sphere: the distinct bins its box c - rmax .. c + rmax touches
// along each axis (periodic; at most (2 rmax + 1) / BINW + 2 <= 17 for the
// radii the 8-bit offset lists allow), then one list entry per bin triple,
// spread over the lanes
constexpr int MAXB = 20;
__global__ void __launch_bounds__(256) k_bins(PDev P, const double* __restrict__ pos, Geom g,
                                              unsigned long long* err, int64_t step) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (a >= P.np) return;
  const double* p = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(p[0], g.nx), nint_idx(p[1], g.ny), nint_idx(p[2], g.nz)};
  const int n[3] = {g.nx, g.ny, g.nz};
  const int nb[3] = {P.nbx, P.nby, P.nbz};
  int bl[3][MAXB], nbl[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d)
    for (int u = c[d] - P.rmax; u <= c[d] + P.rmax; ++u) {
      int bin = (wrap1(u, n[d]) - 1) / BINW;
      bool seen = false;
      for (int k = 0; k < nbl[d]; ++k) seen |= (bl[d][k] == bin);
      if (!seen && nbl[d] < MAXB) bl[d][nbl[d]++] = bin;
    }
  const int total = nbl[0] * nbl[1] * nbl[2];
  for (int t = lane; t < total; t += 32) {
    const int bi = t % nbl[0], bj = (t / nbl[0]) % nbl[1], bk = t / (nbl[0] * nbl[1]);
    const int bin = bl[0][bi] + nb[0] * (bl[1][bj] + nb[1] * bl[2][bk]);
    const int slot = atomicAdd(P.bin_cnt + bin, 1);
    if (slot < BIN_CAP) P.bin_list[size_t(bin) * BIN_CAP + slot] = a;
    else raise_error(err, LBX_DEV_LIST_OVERFLOW, step, a);
  }
}

// ascending particle order inside each bin (the first-match rules below then
// pick the lowest index deterministically)
__global__ void k_bins_sort(PDev P, int nbins) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  int n = min(P.bin_cnt[b], BIN_CAP);
  int* L = P.bin_list + size_t(b) * BIN_CAP;
  for (int i = 1; i < n; ++i) {
    int v = L[i], j = i - 1;
    while (j >= 0 && L[j] > v) { L[j + 1] = L[j]; --j; }
    L[j + 1] = v;
  }
}

__device__ __forceinline__ int bin_of(const PDev& P, int x0, int y0, int z0) {  // 0-based cell coords
  return (x0 / BINW) + P.nbx * ((y0 / BINW) + P.nby * (z0 / BINW));
}

// init_isfluid_CG: flags of the current step and the owning sphere.  A cell
// takes the template value of the lowest-index sphere whose template holds it
// (the reference's first match over its ascending particle lists).  Two
// passes over the solid template cells of every sphere: the owner as an
// atomic minimum (owner and flags start at -1 / fluid), then the owner's
// template value.
__global__ void __launch_bounds__(256) k_stamp(PDev P, const double* __restrict__ pos, Geom g) {
  const int a = blockIdx.x;
  const double* p = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(p[0], g.nx), nint_idx(p[1], g.ny), nint_idx(p[2], g.nz)};
  const int nn[3] = {g.nx, g.ny, g.nz};
  const bool inside = box_inside(P, g, c);
  __shared__ int tiles[12];  // the sphere's tile ranges, once per CTA
  if (P.exact_tiles) {
    if (threadIdx.x == 0) tile_ranges(p, nn, P.rdim, tiles);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < P.n_solid; t += blockDim.x) {
    int dx, dy, dz, v, i1, j1, k1;
    unpack_off(P.offs[t], dx, dy, dz, v);
    if (!offset_cell_in(P, g, inside, c, dx, dy, dz, i1, j1, k1)) continue;
    if (P.exact_tiles && !in_tile_ranges(tiles, (i1 - 1) / TILEX + 1, (j1 - 1) / TILEY + 1, (k1 - 1) / TILEZ + 1))
      continue;
    atomicMin(reinterpret_cast<unsigned*>(P.owner) + cell0(g, i1, j1, k1), unsigned(a));
  }
}

__global__ void __launch_bounds__(256) k_stamp_flags(PDev P, const double* __restrict__ pos, Geom g,
                                                     int8_t* __restrict__ flags_new) {
  const int a = blockIdx.x;
  const double* p = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(p[0], g.nx), nint_idx(p[1], g.ny), nint_idx(p[2], g.nz)};
  const bool inside = box_inside(P, g, c);
  for (int t = threadIdx.x; t < P.n_solid; t += blockDim.x) {
    int dx, dy, dz, v, i1, j1, k1;
    unpack_off(P.offs[t], dx, dy, dz, v);
    if (!offset_cell_in(P, g, inside, c, dx, dy, dz, i1, j1, k1)) continue;
    const int cell = cell0(g, i1, j1, k1);
    if (P.owner[cell] == a) flags_new[cell] = int8_t(v);
  }
}

// Undo a stamping: every solid template cell of the spheres at `pos` back to
// fluid (flags) and to no owner.  Flags and owners are otherwise fluid / -1,
// so clearing what the last stamping at these positions touched restores the
// whole array without a full pass over the lattice.
__global__ void __launch_bounds__(256) k_unstamp(PDev P, const double* __restrict__ pos, Geom g, int8_t* flags,
                                                 int* owner) {
  const int a = blockIdx.x;
  const double* p = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(p[0], g.nx), nint_idx(p[1], g.ny), nint_idx(p[2], g.nz)};
  const bool inside = box_inside(P, g, c);
  for (int t = threadIdx.x; t < P.n_solid; t += blockDim.x) {
    int dx, dy, dz, v, i1, j1, k1;
    unpack_off(P.offs[t], dx, dy, dz, v);
    if (!offset_cell_in(P, g, inside, c, dx, dy, dz, i1, j1, k1)) continue;
    const int cell = cell0(g, i1, j1, k1);
    if (flags) flags[cell] = LBX_FLUID_FLUID;
    if (owner) owner[cell] = -1;
  }
}

// walk the (2 rmax + 1)^3 box around centre c; fn(i1, j1, k1, di, dj, dk) gets
// 1-based coordinates and the reference's getDelta offset, once per cell
template <typename F>
__device__ __forceinline__ void for_box(const PDev& P, const Geom& g, const int c[3], F&& fn) {
  const int w = 2 * P.rmax + 1, tot = w * w * w;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    int dx = t % w - P.rmax, dy = (t / w) % w - P.rmax, dz = t / (w * w) - P.rmax;
    int i1 = wrap1(c[0] + dx, g.nx), j1 = wrap1(c[1] + dy, g.ny), k1 = wrap1(c[2] + dz, g.nz);
    int di = get_delta(i1, c[0], g.nx, P.rdim), dj = get_delta(j1, c[1], g.ny, P.rdim),
        dk = get_delta(k1, c[2], g.nz, P.rdim);
    if (di != dx || dj != dy || dk != dz) continue;  // visited under its reference offset
    fn(i1, j1, k1, di, dj, dk);
  }
}

__device__ __forceinline__ bool moved(const double* p0, const double* p1) {
  return nint_d(p0[0]) != nint_d(p1[0]) || nint_d(p0[1]) != nint_d(p1[1]) || nint_d(p0[2]) != nint_d(p1[2]);
}

// del_fluid: cells fluid in the previous step and solid now hand their
// momentum (rho u of the streamed populations) to the sphere.
template <typename S>
__global__ void __launch_bounds__(256) k_drain(PDev P, const double* __restrict__ pos_cur,
                                               const double* __restrict__ pos_old, double* acc, const S* A,
                                               const S* Bold, Geom g, Shift<typename Store<S>::C> sh,
                                               const int8_t* __restrict__ fold, const int8_t* __restrict__ fnew,
                                               const typename Store<S>::C* __restrict__ rhoR,
                                               const typename Store<S>::C* __restrict__ rhoB) {
  using C = typename Store<S>::C;
  const int a = blockIdx.x;
  const double* pc = pos_cur + size_t(a) * PS;
  const double* po = pos_old + size_t(a) * PS;
  if (!moved(pc, po)) return;
  const int c[3] = {nint_idx(po[0], g.nx), nint_idx(po[1], g.ny), nint_idx(po[2], g.nz)};
  const int n[3] = {g.nx, g.ny, g.nz};
  double s[6] = {0, 0, 0, 0, 0, 0};
  for_box(P, g, c, [&](int i1, int j1, int k1, int di, int dj, int dk) {
    if (di * di + dj * dj + dk * dk > P.sphereMax) return;
    if (P.exact_tiles &&
        !tile_covered(pc, n, P.rdim, (i1 - 1) / TILEX + 1, (j1 - 1) / TILEY + 1, (k1 - 1) / TILEZ + 1))
      return;
    int cell = cell0(g, i1, j1, k1);
    int8_t fo = fold[cell], fn = fnew[cell];
    if (fo != LBX_FLUID_FLUID || (fn != LBX_FLUID_SPHERELIST && fn != LBX_FLUID_SPHEREDEAD)) return;
    Nbr b;
    make_nbr(g, i1 - 1, j1 - 1, k1 - 1, b);
    C qR[Q], qB[Q];
    pull_dead(A, Bold, g, b, 0, sh, fold, qR);
    pull_dead(A, Bold, g, b, 1, sh, fold, qB);
    if (sh.sd) sd_to_rb(qR, qB);  // sum / difference pairs: the components' momenta below
    C rR = rhoR[2 * size_t(cell)], rB = rhoB[2 * size_t(cell)];
    C invrho = C(1) / (rR + rB);
    C u = invrho * mx(qR) + invrho * mx(qB);
    C v = invrho * my(qR) + invrho * my(qB);
    C w = invrho * mz(qR) + invrho * mz(qB);
    double ft[3] = {double((rR + rB) * u), double((rR + rB) * v), double((rR + rB) * w)};
    s[0] += ft[0]; s[1] += ft[1]; s[2] += ft[2];
    if (P.lrotate) {
      double r[3], t[3];
      lever(g, pc, i1, j1, k1, fn == LBX_FLUID_SPHERELIST, P.rdim, r);
      cross(r, ft, t);
      s[3] += t[0]; s[4] += t[1]; s[5] += t[2];
    }
  });
  double out[6] = {0, 0, 0, 0, 0, 0};
  block_sum<6>(s, out);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      acc[size_t(a) * AS + 6 + d] += out[d];
      acc[size_t(a) * AS + 9 + d] += out[3 + d];
    }
}

// init_rho*_CG with flags: densities and phase field of every cell
template <typename S>
__global__ void __launch_bounds__(256) k_rho_p(const S* __restrict__ A, const S* Bold, Geom g,
                                               Shift<typename Store<S>::C> sh, const int8_t* __restrict__ fold,
                                               const int8_t* __restrict__ fnew, typename Store<S>::C* phi,
                                               typename Store<S>::C* rhoR, typename Store<S>::C* rhoB,
                                               unsigned long long* err, int64_t step) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C rR = 0, rB = 0;
  if (fnew[cell] == LBX_FLUID_FLUID) {
    C f[Q];
    pull_dead(A, Bold, g, b, 0, sh, fold, f);
    rR = sum_q(f);
    pull_dead(A, Bold, g, b, 1, sh, fold, f);
    rB = sum_q(f);
    if (sh.sd) {  // sum / difference pairs: rho and rhoR - rhoB
      const C t = rR;
      rR = C(0.5) * (t + rB);
      rB = C(0.5) * (t - rB);
    }
    if (rR < C(-10) || rR > C(10) || rB < C(-10) || rB > C(10)) raise_error(err, LBX_DEV_RHO_RANGE, step, cell);
    if (rR < C(0)) rR = C(0);
    if (rB < C(0)) rB = C(0);
  }
  rhoR[2 * size_t(cell)] = rR;
  rhoB[2 * size_t(cell)] = rB;
  phi[cell] = (rR - rB) / (rR + rB);
}

// both components of one direction and cell (adjacent in memory), one load
__device__ __forceinline__ void ld_pair(const float* p, float, float, float& a, float& b) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ld_pair(const double* p, double, double, double& a, double& b) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ld_pair(const __half* p, float s0, float s1, float& a, float& b) {
  const float2 v = __half22float2(__ldg(reinterpret_cast<const __half2*>(p)));
  a = v.x + s0;
  b = v.y + s1;
}
__device__ __forceinline__ void ld_pair(const __nv_bfloat16* p, float s0, float s1, float& a, float& b) {
  const float2 v = __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162*>(p)));
  a = v.x + s0;
  b = v.y + s1;
}

// clamped densities of a cell fluid in both steps, pulled (init_rho*_CG; a
// cell fluid in the previous step has no spheredead source); the sums run
// over the directions in order, as init_rhoR_CG / init_rhoB_CG do
template <typename S, typename C = typename Store<S>::C>
__device__ __forceinline__ void pulled_rho(const S* A, const Geom& g, const Shift<C>& sh, int i1, int j1, int k1,
                                           C& rR, C& rB) {
  Nbr b;
  make_nbr(g, i1 - 1, j1 - 1, k1 - 1, b);
  C fR[Q], fB[Q];
#pragma unroll
  for (int l = 0; l < Q; ++l)
    ld_pair(A + pidx(g, 0, l, at(b, -ex(l), -ey(l), -ez(l))), sh.at(0, l), sh.at(1, l), fR[l], fB[l]);
  rR = sum_q(fR);
  rB = sum_q(fB);
  if (sh.sd) {  // sum / difference pairs: rho and rhoR - rhoB
    const C t = rR;
    rR = C(0.5) * (t + rB);
    rB = C(0.5) * (t - rB);
  }
  rR = rR < C(0) ? C(0) : rR;
  rB = rB < C(0) ? C(0) : rB;
}

// init_rho*_CG for the fluid cells around each sphere (single-pass schedule).
// The particle kernels are the only readers of the densities of fluid cells
// (the fluid kernel pulls its own), and they read them within
// (rdim + sqrt 3) of a sphere's centre: the bounce-back of this step at the
// fluid end of each surface link, the wetting and fill kernels in the first
// (D3Q27) belt of a surface or uncovered cell, the drain of the next step at
// the cells the spheres then cover: all of them fluid cells with a D3Q27
// neighbour in the template.  The shell is that belt (and the template cells
// the tile-list coverage may have left fluid) around the current centre and,
// for a sphere that changed cell, around the previous one (its uncovered
// cells).  The rare second-belt fallbacks pull their own.
template <typename S>
__global__ void __launch_bounds__(256) k_rho_shell(PDev P, const double* __restrict__ pos_cur,
                                                   const double* __restrict__ pos_old, const S* A, Geom g,
                                                   Shift<typename Store<S>::C> sh, const int8_t* __restrict__ fold,
                                                   const int8_t* __restrict__ fnew, typename Store<S>::C* rhoR,
                                                   typename Store<S>::C* rhoB) {
  using C = typename Store<S>::C;
  // spheres in reverse order: the bounce-back before this kernel (the end of
  // the previous step) rewrote the belts' links sphere by sphere in
  // ascending order, so the last ones are still in L2 (the values do not
  // depend on the order: a cell in two belts gets the same sums)
  const int a = P.np - 1 - int(blockIdx.x);
  const double* pc = pos_cur + size_t(a) * PS;
  const double* po = pos_old + size_t(a) * PS;
  const int cn[3] = {nint_idx(pc[0], g.nx), nint_idx(pc[1], g.ny), nint_idx(pc[2], g.nz)};
  const int co[3] = {nint_idx(po[0], g.nx), nint_idx(po[1], g.ny), nint_idx(po[2], g.nz)};
  const bool mv = moved(pc, po);
  const int tot = mv ? 2 * P.n_shell : P.n_shell;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const bool second = t >= P.n_shell;
    int dx, dy, dz, tv;
    unpack_off(P.offs_shell[second ? t - P.n_shell : t], dx, dy, dz, tv);
    // around the old centre too (its uncovered cells' belt); a cell near
    // both centres is summed twice, with the same result
    const int* c0 = second ? co : cn;
    const int i1 = wrap1(c0[0] + dx, g.nx), j1 = wrap1(c0[1] + dy, g.ny), k1 = wrap1(c0[2] + dz, g.nz);
    const int y = cell0(g, i1, j1, k1);
    // outside the sphere's own template the cell is nearly always fluid: the
    // flags and the pull are loaded together, the pull dropped if unused
    const int8_t fn = fnew[y], fo = fold[y];
    if (tv != LBX_FLUID_FLUID && (fn != LBX_FLUID_FLUID || fo != LBX_FLUID_FLUID)) continue;
    C rR, rB;
    pulled_rho(A, g, sh, i1, j1, k1, rR, rB);
    if (fn != LBX_FLUID_FLUID || fo != LBX_FLUID_FLUID) continue;
    rhoR[2 * size_t(y)] = rR;
    rhoB[2 * size_t(y)] = rB;
  }
}

// make_fluid: cells solid in the previous step and fluid now get the mean
// density of their fluid neighbours (D3Q27 belt, then the 98-cell second
// belt) and the equilibrium at the sphere's velocity; the sphere pays the
// momentum.  The populations go where the fluid step reads them: with the
// two-pass schedule into B at the cell (its collision reads a new cell
// there), with the single-pass kernel (pulls != nullptr, the populations A
// of this step) into the slots the cell pulls from, A(l, x - e_l): only cell
// x pulls each of them, so the fluid kernel needs no case for new cells.
template <typename S>
__global__ void __launch_bounds__(256) k_fill(PDev P, const double* __restrict__ pos_cur,
                                              const double* __restrict__ pos_old, double* acc, const S* A, S* B,
                                              S* pulls, Geom g, Shift<typename Store<S>::C> sh,
                                              LatticeT<typename Store<S>::C> L, const int8_t* __restrict__ fold,
                                              const int8_t* __restrict__ fnew, typename Store<S>::C* rhoR,
                                              typename Store<S>::C* rhoB, typename Store<S>::C* phi) {
  using C = typename Store<S>::C;
  const int a = blockIdx.x;
  const double* pc = pos_cur + size_t(a) * PS;
  const double* po = pos_old + size_t(a) * PS;
  if (!moved(pc, po)) return;
  const int c[3] = {nint_idx(po[0], g.nx), nint_idx(po[1], g.ny), nint_idx(po[2], g.nz)};
  const int n[3] = {g.nx, g.ny, g.nz};
  double s[6] = {0, 0, 0, 0, 0, 0};
  for_box(P, g, c, [&](int i1, int j1, int k1, int di, int dj, int dk) {
    if (di * di + dj * dj + dk * dk > P.sphereMax) return;
    if (P.exact_tiles &&
        !tile_covered(pc, n, P.rdim, (i1 - 1) / TILEX + 1, (j1 - 1) / TILEY + 1, (k1 - 1) / TILEZ + 1))
      return;
    int cell = cell0(g, i1, j1, k1);
    int8_t fo = fold[cell], fn = fnew[cell];
    if ((fo != LBX_FLUID_SPHERELIST && fo != LBX_FLUID_SPHEREDEAD) || fn != LBX_FLUID_FLUID) return;
    C Rs = 0, Bs = 0;
    int D = 0;
    for (int l = 1; l < Q27; ++l) {  // compute_onebelt_density_twofluids
      int yi = wrap1(i1 + ex27(l), g.nx), yj = wrap1(j1 + ey27(l), g.ny), yk = wrap1(k1 + ez27(l), g.nz);
      int y = cell0(g, yi, yj, yk);
      if (fnew[y] == LBX_FLUID_FLUID && fold[y] == LBX_FLUID_FLUID) {
        Rs = Rs + rhoR[2 * size_t(y)]; Bs = Bs + rhoB[2 * size_t(y)]; ++D;
      }
    }
    if (D) { Rs = Rs / C(D); Bs = Bs / C(D); }
    else {  // compute_secbelt_density_twofluids
      Rs = 0; Bs = 0;
      for (int kk = -2; kk <= 2; ++kk)
        for (int jj = -2; jj <= 2; ++jj)
          for (int ii = -2; ii <= 2; ++ii) {
            if (!(ii == -2 || ii == 2 || jj == -2 || jj == 2 || kk == -2 || kk == 2)) continue;
            int yi = wrap1(i1 + ii, g.nx), yj = wrap1(j1 + jj, g.ny), yk = wrap1(k1 + kk, g.nz);
            int y = cell0(g, yi, yj, yk);
            if (fnew[y] == LBX_FLUID_FLUID && fold[y] == LBX_FLUID_FLUID) {
              C qR, qB;
              pulled_rho(A, g, sh, yi, yj, yk, qR, qB);  // beyond the density shell
              Rs = Rs + qR; Bs = Bs + qB; ++D;
            }
          }
      if (D) { Rs = Rs / C(D); Bs = Bs / C(D); }
      // else fix_onebelt_density_twofluids (empty in the reference): zero density
    }
    C u = C(pc[3]), v = C(pc[4]), w = C(pc[5]);
    rhoR[2 * size_t(cell)] = Rs;
    rhoB[2 * size_t(cell)] = Bs;
    phi[cell] = (Rs - Bs) / (Rs + Bs);
    C usq = L.half_inv_cssq * (u * u + v * v + w * w);
    Nbr b;
    make_nbr(g, i1 - 1, j1 - 1, k1 - 1, b);
    for (int comp = 0; comp < 2; ++comp) {
      // sum / difference pairs store the equilibria of rho and rhoR - rhoB
      C r = sh.sd ? (comp ? Rs - Bs : Rs + Bs) : (comp ? Bs : Rs);
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        S* dst = pulls ? pulls + pidx(g, comp, l, at(b, -ex(l), -ey(l), -ez(l))) : B + pidx(g, comp, l, cell);
        Store<S>::st(dst, equil_u(L, r, edot(l, u, v, w), usq, l), sh.at(comp, l));
      }
    }
    double ft[3] = {double(-(Rs + Bs) * u), double(-(Rs + Bs) * v), double(-(Rs + Bs) * w)};
    s[0] += ft[0]; s[1] += ft[1]; s[2] += ft[2];
    if (P.lrotate) {
      double r[3], t[3];
      lever(g, pc, i1, j1, k1, fo == LBX_FLUID_SPHERELIST, P.rdim, r);
      cross(r, ft, t);
      s[3] += t[0]; s[4] += t[1]; s[5] += t[2];
    }
  });
  double out[6] = {0, 0, 0, 0, 0, 0};
  block_sum<6>(s, out);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      acc[size_t(a) * AS + 6 + d] += out[d];
      acc[size_t(a) * AS + 9 + d] += out[3 + d];
    }
}

// virtual densities of the surface cells a sphere owns: Janus
// (compute_virtual_rho) or neutral wetting (compute_densities_wall)
template <typename S, typename C = typename Store<S>::C>
__global__ void __launch_bounds__(256, 3) k_virtual(PDev P, const double* __restrict__ pos, Geom g, int neutral,
                                                 const S* A, Shift<C> sh,
                                                 const int8_t* __restrict__ fold, const int8_t* __restrict__ fnew,
                                                 C* rhoR, C* rhoB, C* phi, LatticeT<C> L) {
  const int a = blockIdx.x;
  const double* pc = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(pc[0], g.nx), nint_idx(pc[1], g.ny), nint_idx(pc[2], g.nz)};
  double xl[3] = {0, 0, 0};
  if (!neutral) {
    double ax[3] = {1.0, 0.0, 0.0};
    to_lab(pc, ax, xl);
  }
  // the cells a sphere owns as surface cells are surface cells of its template
  for (int t = threadIdx.x; t < P.n_surf; t += blockDim.x) {
    int dx, dy, dz, tv, i1, j1, k1;
    unpack_off(P.offs[t], dx, dy, dz, tv);
    if (!offset_cell(P, g, c, dx, dy, dz, i1, j1, k1)) continue;
    int cell = cell0(g, i1, j1, k1);
    if (fnew[cell] != LBX_FLUID_SPHERELIST || P.owner[cell] != a) continue;
    C R, Bv;
    if (!neutral) {
      double r[3] = {double(i1) - pc[0], double(j1) - pc[1], double(k1) - pc[2]};
      r[0] = r[0] - double(g.nx) * double(nint_d((1.0 / g.nx) * r[0]));
      r[1] = r[1] - double(g.ny) * double(nint_d((1.0 / g.ny) * r[1]));
      r[2] = r[2] - double(g.nz) * double(nint_d((1.0 / g.nz) * r[2]));
      double m = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      double cs = xl[0] * (r[0] / m) + xl[1] * (r[1] / m) + xl[2] * (r[2] / m);
      if (cs < 0.0) { R = 0; Bv = 1; }
      else { R = 1; Bv = 0; }
    } else {
      // compute_onebelt_density_2fl_weights, nine neighbours at a time (the
      // periodic rows and planes of the cell from make_nbr): their flags, the
      // fluid ones' densities, then the sums in ascending direction order
      Nbr b;
      make_nbr(g, i1 - 1, j1 - 1, k1 - 1, b);
      C Rs = 0, Bs = 0, Ds = 0;
#pragma unroll
      for (int l0 = 1; l0 < Q27; l0 += 9) {
        bool fl[9];
        C vr[9], vb[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const int l = l0 + k;
          fl[k] = l < Q27 && fnew[at(b, ex27(l), ey27(l), ez27(l))] == LBX_FLUID_FLUID;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const int l = l0 + k;
          vr[k] = vb[k] = C(0);
          if (l < Q27 && fl[k]) ld_two(rhoR + 2 * size_t(at(b, ex27(l), ey27(l), ez27(l))), vr[k], vb[k]);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const int l = l0 + k;
          if (l < Q27 && fl[k]) {
            C w = L.p27[wclass27(l)];
            Rs = Rs + w * vr[k]; Bs = Bs + w * vb[k]; Ds = Ds + w;
          }
        }
      }
      if (Ds != C(0)) { R = Rs / Ds; Bv = Bs / Ds; }
      else {
        int D = 0;
        Rs = 0; Bs = 0;
        for (int kk = -2; kk <= 2; ++kk)
          for (int jj = -2; jj <= 2; ++jj)
            for (int ii = -2; ii <= 2; ++ii) {
              if (!(ii == -2 || ii == 2 || jj == -2 || jj == 2 || kk == -2 || kk == 2)) continue;
              int yi = wrap1(i1 + ii, g.nx), yj = wrap1(j1 + jj, g.ny), yk = wrap1(k1 + kk, g.nz);
              int y = cell0(g, yi, yj, yk);
              if (fnew[y] == LBX_FLUID_FLUID && fold[y] == LBX_FLUID_FLUID) {
                C qR, qB;
                pulled_rho(A, g, sh, yi, yj, yk, qR, qB);  // beyond the density shell
                Rs = Rs + qR; Bs = Bs + qB; ++D;
              }
            }
        // no fluid in either belt: the density stays at init_rho*_CG's zero
        R = D ? Rs / C(D) : C(0);
        Bv = D ? Bs / C(D) : C(0);
      }
    }
    rhoR[2 * size_t(cell)] = R;
    rhoB[2 * size_t(cell)] = Bv;
    phi[cell] = (R - Bv) / (R + Bv);
  }
}

// time_step_CG with flags (two-pass schedule): collision on fluid cells,
// the streamed populations pass through unchanged elsewhere.
template <typename S, bool DD>
__global__ void __launch_bounds__(256) k_collide_p(const S* __restrict__ A, S* B, Geom g,
                                                   Shift<typename Store<S>::C> sh,
                                                   const typename Store<S>::C* __restrict__ phi,
                                                   const typename Store<S>::C* __restrict__ rhoR,
                                                   const typename Store<S>::C* __restrict__ rhoB,
                                                   const int8_t* __restrict__ fold, const int8_t* __restrict__ fnew,
                                                   CGConst<typename Store<S>::C> K) {
  using C = typename Store<S>::C;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  Nbr b;
  make_nbr(g, x, y, z, b);
  int cell = at(b, 0, 0, 0);
  C fR[Q], fB[Q];
  int8_t fn = fnew[cell];
  bool fresh = (fn == LBX_FLUID_FLUID) && (fold[cell] != LBX_FLUID_FLUID);
  if (fresh) {  // make_fluid already wrote the new node's populations into B
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      fR[l] = Store<S>::ld(B + pidx(g, 0, l, cell), sh.at(0, l));
      fB[l] = Store<S>::ld(B + pidx(g, 1, l, cell), sh.at(1, l));
    }
  } else {
    pull_dead(A, B, g, b, 0, sh, fold, fR);
    pull_dead(A, B, g, b, 1, sh, fold, fB);
  }
  if (fn == LBX_FLUID_FLUID) {
    C psix, psiy, psiz;
    if constexpr (DD) {  // two fluid densities: gradients from the density arrays
      C psR[3], psB[3];
      grad27_dd(
          K,
          [&](int dx, int dy, int dz, C& rs, C& bs) {
            const int y = at(b, dx, dy, dz);
            rs = rhoR[2 * size_t(y)];
            bs = rhoB[2 * size_t(y)];
          },
          psix, psiy, psiz, psR, psB);
      cg_collide_cell_dd(K, fR, fB, rhoR[2 * size_t(cell)], rhoB[2 * size_t(cell)], psix, psiy, psiz, psR, psB);
    } else {
      grad27(K.L, [&](int dx, int dy, int dz) { return phi[at(b, dx, dy, dz)]; }, psix, psiy, psiz);
      cg_collide_cell(K, fR, fB, rhoR[2 * size_t(cell)], rhoB[2 * size_t(cell)], psix, psiy, psiz);
    }
  }
  store_all(B, g, cell, 0, sh, fR);
  store_all(B, g, cell, 1, sh, fB);
}

// one bounce-back link of sphere a at surface cell (i1,j1,k1):
// returns the force / torque of node_to_particle_bounce_back_bc2 and, when
// `wall` is given, the moving-wall terms of phase 2.
struct LinkGeo {
  double rv[3], ol[3];
};

// lab-frame angular velocity of a sphere (zero without rotation)
__device__ __forceinline__ void lab_omega(const PDev& P, const double* pc, double ol[3]) {
  ol[0] = ol[1] = ol[2] = 0;
  if (P.lrotate) {
    double om[3] = {pc[6], pc[7], pc[8]};
    to_lab(pc, om, ol);
  }
}

__device__ __forceinline__ void link_geo(const PDev& P, const Geom& g, const double* pc, int i1, int j1, int k1,
                                         LinkGeo& G) {
  G.rv[0] = G.rv[1] = G.rv[2] = 0;
  lab_omega(P, pc, G.ol);
  if (P.lrotate) lever(g, pc, i1, j1, k1, true, P.rdim, G.rv);
}

// the same with the sphere's lab angular velocity already known
__device__ __forceinline__ void link_geo_ol(const PDev& P, const Geom& g, const double* pc, const double ol[3], int i1,
                                            int j1, int k1, LinkGeo& G) {
  G.rv[0] = G.rv[1] = G.rv[2] = 0;
  G.ol[0] = ol[0];
  G.ol[1] = ol[1];
  G.ol[2] = ol[2];
  if (P.lrotate) lever(g, pc, i1, j1, k1, true, P.rdim, G.rv);
}

// the same for a cell at offset d of the sphere's own offset lists: the
// minimum image of (cell - centre) is d + (nint(centre) - centre), so the
// lever needs no image division
__device__ __forceinline__ void own_link_geo(const PDev& P, const double* pc, const int c[3], const double ol[3],
                                             int dx, int dy, int dz, LinkGeo& G) {
  G.rv[0] = G.rv[1] = G.rv[2] = 0;
  G.ol[0] = ol[0];
  G.ol[1] = ol[1];
  G.ol[2] = ol[2];
  if (P.lrotate) {
    double r[3] = {double(dx) + (double(c[0]) - pc[0]), double(dy) + (double(c[1]) - pc[1]),
                   double(dz) + (double(c[2]) - pc[2])};
    const double m = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int d = 0; d < 3; ++d) G.rv[d] = P.rdim / m * r[d];
  }
}

__device__ __forceinline__ void wall_velocity(const PDev& P, const double* pc, const LinkGeo& G, int lr,
                                              double rt[3], double v[3]) {
  v[0] = pc[3]; v[1] = pc[4]; v[2] = pc[5];
  rt[0] = rt[1] = rt[2] = 0;
  if (P.lrotate) {
    rt[0] = G.rv[0] + 0.5 * ex(lr);
    rt[1] = G.rv[1] + 0.5 * ey(lr);
    rt[2] = G.rv[2] + 0.5 * ez(lr);
    double c[3];
    cross(G.ol, rt, c);
    v[0] += c[0]; v[1] += c[1]; v[2] += c[2];
  }
}

// partBB_CG + partBB_CG_p2n + partBB_CG_p2n2.  A thread takes one surface
// cell within the sphere's reach.  The links that cross the surface are found
// first (at most one per opposite pair), the populations and densities of
// their fluid ends are loaded together, then: the node -> particle momentum
// of this sphere; and, for the cell's owner only, the bounce-back copy and
// the moving-wall corrections of every sphere in reach (ascending index, each
// rounded to the storage type as a store and reload would), kept in
// registers and stored once.  mode selects the phases (BB_N2P | BB_COPY |
// BB_WALL; the step runs all three in one launch, the kernel-level entry
// points one each, with the same results).
constexpr int BB_N2P = 1, BB_COPY = 2, BB_WALL = 4, BB_ALL = 7;

// Whether another sphere's template can reach into the bounce-back reach of
// sphere a (offsets d^2 < sphereMax around its rounded centre c): such a
// sphere has a template cell inside a's box, so it is listed in one of the
// bins of a's box, and its rounded centre lies within the bound below
// (minimum image).  With rmax <= BINW the box spans at most three bins per axis, those
// of c - rmax, c and c + rmax; larger radii answer yes.  A vote of the calling
// warp (lanes 0..26 take one bin each; no CTA barrier), called by all its
// lanes.
__device__ bool crowded_reach(const PDev& P, const double* __restrict__ pos, const Geom& g, int a, const int c[3]) {
  bool hit = P.rmax > BINW;
  const int t = threadIdx.x & 31;
  if (!hit && t < 27) {
    const int s[3] = {(t % 3 - 1) * P.rmax, ((t / 3) % 3 - 1) * P.rmax, (t / 9 - 1) * P.rmax};
    const int x0 = wrap1(c[0] + s[0], g.nx) - 1, y0 = wrap1(c[1] + s[1], g.ny) - 1, z0 = wrap1(c[2] + s[2], g.nz) - 1;
    const int bin = bin_of(P, x0, y0, z0);
    const int cnt = min(P.bin_cnt[bin], BIN_CAP);
    const int* L = P.bin_list + size_t(bin) * BIN_CAP;
    const int n[3] = {g.nx, g.ny, g.nz};
    // a template cell of q (|o|^2 <= rdim^2) inside a's reach (|r|^2 <
    // sphereMax): |c_q - c| = |r - o| < rdim + sqrt(sphereMax)
    const double lim_r = P.rdim + sqrt(double(P.sphereMax));
    const double lim = lim_r * lim_r;
    for (int u = 0; u < cnt && !hit; ++u) {
      const int q = L[u];
      if (q == a) continue;
      const double* pq = pos + size_t(q) * PS;
      const int cq[3] = {nint_idx(pq[0], g.nx), nint_idx(pq[1], g.ny), nint_idx(pq[2], g.nz)};
      int d2 = 0;
      for (int d = 0; d < 3; ++d) {
        int v = cq[d] - c[d];
        v -= n[d] * int(floorf(float(v) / float(n[d]) + 0.5f));  // minimum image
        d2 += v * v;
      }
      hit = double(d2) < lim;
    }
  }
  return __any_sync(0xffffffffu, hit);
}

// the vote once per sphere, after the lists are built (one warp per sphere),
// so that the bounce-back starts from one byte instead of the bins
__global__ void __launch_bounds__(256) k_crowd(PDev P, const double* __restrict__ pos, Geom g) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (a >= P.np) return;  // whole warps: np * 32 threads, rounded up to full CTAs
  const double* p = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(p[0], g.nx), nint_idx(p[1], g.ny), nint_idx(p[2], g.nz)};
  const bool hit = crowded_reach(P, pos, g, a, c);
  if ((threadIdx.x & 31) == 0) P.crowd[a] = int8_t(hit);
}

template <typename S>
__global__ void __launch_bounds__(256, sizeof(S) == 8 ? 1 : 2) k_bb(PDev P, const double* __restrict__ pos, double* acc, S* B, Geom g,
                                            Shift<typename Store<S>::C> sh, LatticeT<typename Store<S>::C> L,
                                            const int8_t* __restrict__ fnew,
                                            const typename Store<S>::C* __restrict__ rhoR,
                                            const typename Store<S>::C* __restrict__ rhoB, int mode) {
  using C = typename Store<S>::C;
  using St = Store<S>;
  const int a = blockIdx.x;
  const double* pc = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(pc[0], g.nx), nint_idx(pc[1], g.ny), nint_idx(pc[2], g.nz)};
  const int nn3[3] = {g.nx, g.ny, g.nz};
  const C buz = C(2) / L.cssq;  // pref_bouzidi, dimensions_m.CUF:95
  double ola[3];
  lab_omega(P, pc, ola);
  // the sphere's tile ranges (its tile-list coverage), once per CTA
  __shared__ int tiles[12];
  if (threadIdx.x == 0) tile_ranges(pc, nn3, P.rdim, tiles);
  __syncthreads();
  double s[6] = {0, 0, 0, 0, 0, 0};
  // Past the sphere's own surface cells (pass 0), the reach holds its dead
  // cells and fluid cells, which no link crosses, unless another sphere's
  // template reaches into it: pass 1 runs only then (k_crowd's vote).
  const bool crowd = P.crowd[a] != 0;
  for (int pass = 0; pass < 2; ++pass) {
  if (pass == 1 && !crowd) break;
  const int t0 = pass ? P.n_surf : 0, t1 = pass ? P.n_bb : P.n_surf;
  for (int t = t0 + int(threadIdx.x); t < t1; t += blockDim.x) {
    int dx, dy, dz, tv, i1, j1, k1;
    unpack_off(P.offs_bb[t], dx, dy, dz, tv);
    if (!offset_cell(P, g, c, dx, dy, dz, i1, j1, k1)) continue;
    const int cell = cell0(g, i1, j1, k1);
    const int x0 = i1 - 1, y0 = j1 - 1, z0 = k1 - 1;
    Nbr b;
    make_nbr(g, x0, y0, z0, b);
    // bit l: neighbour l is fluid.  For the sphere's own surface offsets (a
    // surface cell nearly always) the neighbours' flags are loaded together
    // with the cell's flag and owner; for the other offsets only if needed.
    auto nbr_fluid = [&]() {
      unsigned m = 0;
#pragma unroll
      for (int l = 1; l < Q; ++l) m |= unsigned(fnew[at(b, ex(l), ey(l), ez(l))] == LBX_FLUID_FLUID) << l;
      return m;
    };
    const bool likely = tv == LBX_FLUID_SPHERELIST;
    const int8_t fc = fnew[cell];
    const int ow = P.owner[cell];
    unsigned fl = likely ? nbr_fluid() : 0u;
    if (fc != LBX_FLUID_SPHERELIST) continue;
    const int ti = x0 / TILEX + 1, tj = y0 / TILEY + 1, tk = z0 / TILEZ + 1;
    // node -> particle momentum exchange for this sphere (atmDist < sphereMax)
    const bool n2p = (mode & BB_N2P) && dx * dx + dy * dy + dz * dz < P.sphereMax &&
                     (!P.exact_tiles || in_tile_ranges(tiles, ti, tj, tk));
    const bool own = (mode & (BB_COPY | BB_WALL)) && ow == a;
    if (!n2p && !own) continue;
    if (!likely) fl = nbr_fluid();
    // link pair it = (lo, hi) = (2it+1, 2it+2) crosses when exactly one end is
    // fluid; hib: the fluid end is hi (then lf = lo, lr = hi), else lo
    int xf[9];
    unsigned act = 0, hib = 0;
#pragma unroll
    for (int it = 0; it < 9; ++it) {
      const int lo = 2 * it + 1, hi = 2 * it + 2;
      const int xi = at(b, ex(lo), ey(lo), ez(lo)), xo = at(b, ex(hi), ey(hi), ez(hi));
      const bool fi = (fl >> lo) & 1u, fo = (fl >> hi) & 1u;
      xf[it] = fo ? xo : xi;
      act |= unsigned(fi != fo) << it;
      hib |= unsigned(fo) << it;
    }
    if (!act) continue;
    S hR[9], hB[9];
    C rR[9], rB[9];
#pragma unroll
    for (int it = 0; it < 9; ++it) {
      hR[it] = hB[it] = S(0.f);
      rR[it] = rB[it] = C(0);
      if (act >> it & 1) {
        const bool h = hib >> it & 1;
        const int lf = h ? 2 * it + 1 : 2 * it + 2, lr = h ? 2 * it + 2 : 2 * it + 1;
        // the fluid end's population, or (wall phase alone) the copy already in place
        const S* p = (n2p || (mode & BB_COPY)) ? B + pidx(g, 0, lf, xf[it]) : B + pidx(g, 0, lr, cell);
        ld_two(p, hR[it], hB[it]);
        ld_two(rhoR + 2 * size_t(xf[it]), rR[it], rB[it]);  // interleaved densities
        if (sh.sd) {  // sum / difference pairs: the wall term of each half is linear in its density
          const C t = rR[it];
          rR[it] = t + rB[it];
          rB[it] = t - rB[it];
        }
      }
    }
    if (n2p) {
      LinkGeo G;
      own_link_geo(P, pc, c, ola, dx, dy, dz, G);
#pragma unroll
      for (int it = 0; it < 9; ++it) {
        if (!(act >> it & 1)) continue;
        const bool h = hib >> it & 1;
        const int lf = h ? 2 * it + 1 : 2 * it + 2, lr = h ? 2 * it + 2 : 2 * it + 1;
        double rt[3], v[3];
        wall_velocity(P, pc, G, lr, rt, v);
        C ev = C(ex(lf)) * C(v[0]) + C(ey(lf)) * C(v[1]) + C(ez(lf)) * C(v[2]);
        C w = L.w[wclass(lf)];
        C f2pR = C(2) * St::dec(hR[it], sh.at(0, lf)) - w * buz * rR[it] * ev;
        C f2pB = C(2) * St::dec(hB[it], sh.at(1, lf)) - w * buz * rB[it] * ev;
        C f2p = sh.sd ? f2pR : f2pR + f2pB;  // sum / difference pairs: the total is the first half
        double ft[3] = {double(f2p * C(ex(lf))), double(f2p * C(ey(lf))), double(f2p * C(ez(lf)))};
        s[0] += ft[0]; s[1] += ft[1]; s[2] += ft[2];
        if (P.lrotate) {
          double tq[3];
          cross(rt, ft, tq);
          s[3] += tq[0] * abs(ex(lf));
          s[4] += tq[1] * abs(ey(lf));
          s[5] += tq[2] * abs(ez(lf));
        }
      }
    }
    if (!own) continue;
    // p2n phase 1: B(lr, cell) = B(lf, fluid end); lr and lf share their shift
    // p2n phase 2: moving-wall corrections of the spheres in reach
    // A sphere no other template reaches (crowd false) is the only one of
    // its bins within sphereMax of its surface cells: its rounded centre is at
    // least rdim + sqrt(sphereMax) from every other listed centre (minimum
    // image; getDelta's offsets are no shorter), and a surface cell is within
    // rdim of its own.  The walk is then the sphere itself.
    const int bin = crowd ? bin_of(P, x0, y0, z0) : 0;
    const int nlist = !(mode & BB_WALL) ? 0 : crowd ? min(P.bin_cnt[bin], BIN_CAP) : 1;
    const int* Lst = P.bin_list + size_t(bin) * BIN_CAP;
    for (int u = 0; u < nlist; ++u) {
      const int q = crowd ? Lst[u] : a;
      const double* pq = pos + size_t(q) * PS;
      int ei = get_delta(i1, nint_idx(pq[0], g.nx), g.nx, P.rdim),
          ej = get_delta(j1, nint_idx(pq[1], g.ny), g.ny, P.rdim),
          ek = get_delta(k1, nint_idx(pq[2], g.nz), g.nz, P.rdim);
      if (ei * ei + ej * ej + ek * ek >= P.sphereMax) continue;
      if (P.exact_tiles && !(q == a ? in_tile_ranges(tiles, ti, tj, tk) : tile_covered(pq, nn3, P.rdim, ti, tj, tk)))
        continue;
      LinkGeo G;
      if (q == a) own_link_geo(P, pc, c, ola, dx, dy, dz, G);  // (ei, ej, ek) is (dx, dy, dz) here
      else link_geo(P, g, pq, i1, j1, k1, G);
#pragma unroll
      for (int it = 0; it < 9; ++it) {
        if (!(act >> it & 1)) continue;
        const bool h = hib >> it & 1;
        const int lf = h ? 2 * it + 1 : 2 * it + 2, lr = h ? 2 * it + 2 : 2 * it + 1;
        double rt[3], v[3];
        wall_velocity(P, pq, G, lr, rt, v);
        C ev = C(ex(lf)) * C(v[0]) + C(ey(lf)) * C(v[1]) + C(ez(lf)) * C(v[2]);
        C w = L.w[wclass(lf)];
        hR[it] = St::enc(St::dec(hR[it], sh.at(0, lr)) - w * buz * rR[it] * ev, sh.at(0, lr));
        hB[it] = St::enc(St::dec(hB[it], sh.at(1, lr)) - w * buz * rB[it] * ev, sh.at(1, lr));
      }
    }
#pragma unroll
    for (int it = 0; it < 9; ++it) {
      if (!(act >> it & 1)) continue;
      const int lr = (hib >> it & 1) ? 2 * it + 2 : 2 * it + 1;
      S* p = B + pidx(g, 0, lr, cell);
      st_two(p, hR[it], hB[it]);
    }
  }
  }
  double out[6] = {0, 0, 0, 0, 0, 0};
  block_sum<6>(s, out);
  if (threadIdx.x == 0)
    for (int d = 0; d < 6; ++d) acc[size_t(a) * AS + d] += out[d];
}

// The crossing links of the bounce-back: for every surface cell within a
// sphere's reach (the node -> particle predicates of k_bb: flag spherelist,
// d^2 < sphereMax, the tile-list coverage), each opposite pair with exactly
// one fluid end, as (sphere, surface cell, direction from the cell towards
// its fluid end).  This is the link set node_to_particle_bounce_back_bc2
// visits (kernels_fluid_PART.CUF:1929-1941, its DEBUG_N2P record); a
// readback kernel, not part of the step.  Entries past `cap` are counted,
// not written.
__global__ void __launch_bounds__(256) k_links(PDev P, const double* __restrict__ pos, Geom g,
                                               const int8_t* __restrict__ fnew, unsigned long long* count,
                                               long long cap, int* lcell, int8_t* ldir, int* lsph) {
  const int a = blockIdx.x;
  const double* pc = pos + size_t(a) * PS;
  const int c[3] = {nint_idx(pc[0], g.nx), nint_idx(pc[1], g.ny), nint_idx(pc[2], g.nz)};
  const int nn3[3] = {g.nx, g.ny, g.nz};
  for (int t = threadIdx.x; t < P.n_bb; t += blockDim.x) {
    int dx, dy, dz, tv, i1, j1, k1;
    unpack_off(P.offs_bb[t], dx, dy, dz, tv);
    if (dx * dx + dy * dy + dz * dz >= P.sphereMax) continue;
    if (!offset_cell(P, g, c, dx, dy, dz, i1, j1, k1)) continue;
    const int cell = cell0(g, i1, j1, k1);
    if (fnew[cell] != LBX_FLUID_SPHERELIST) continue;
    const int x0 = i1 - 1, y0 = j1 - 1, z0 = k1 - 1;
    if (P.exact_tiles && !tile_covered(pc, nn3, P.rdim, x0 / TILEX + 1, y0 / TILEY + 1, z0 / TILEZ + 1)) continue;
    Nbr b;
    make_nbr(g, x0, y0, z0, b);
    for (int it = 0; it < 9; ++it) {
      const int lo = 2 * it + 1, hi = 2 * it + 2;
      const bool fi = fnew[at(b, ex(lo), ey(lo), ez(lo))] == LBX_FLUID_FLUID;
      const bool fo = fnew[at(b, ex(hi), ey(hi), ez(hi))] == LBX_FLUID_FLUID;
      if (fi == fo) continue;
      const unsigned long long k = atomicAdd(count, 1ull);
      if ((long long)k < cap) {
        lcell[k] = cell;
        ldir[k] = int8_t(fo ? hi : lo);
        lsph[k] = a;
      }
    }
  }
}

// inter_force_particles / addHertzian: all pairs; one warp per sphere, the
// lanes take every 32nd partner and the warp sums their shares in a fixed
// order.  With lubrication on, the analytic squeeze force is added as well
// (the reference writes it into a total that its integrator then
// overwrites; here it reaches the integrator).  With the learned closure the
// same pass lists each sphere's close partners for it (nbr, cnt), so the
// closure costs no second all-pairs pass.
__global__ void __launch_bounds__(256) k_pairs(PDev P, const double* __restrict__ pos, double* acc, Geom g,
                                               double gap_cut, int* nbr, int* cnt, unsigned long long* err,
                                               int64_t step) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= P.np) return;
  const double rsqcut = P.hz_rmin * P.hz_rmin;
  const double gmin = 5.0 * 0.5 * P.hz_k * pow(P.hz_rmin - P.hz_rcap, 1.5);
  const double rpar = 2.0 * P.rdim;
  const double lubfactor = P.lub_k * 6.0 * 3.141592653589793238462643383279502884 * pow(P.rdim * P.rdim, 2.0) / (rpar * rpar);
  const double rparcut = rpar + P.lub_rmin;
  const double mxrsqcut = fmax(rparcut * rparcut, rsqcut);
  const double rparcap = rpar + P.lub_rcap;
  // closure neighbour list (nbr != nullptr): partners with gap below gap_cut,
  // ascending (32 partners per pass, hits appended in lane order)
  const double nbr_pre = (2.0 * P.rdim + gap_cut + 1.0) * (2.0 * P.rdim + gap_cut + 1.0);
  double f[3] = {0, 0, 0}, fl[3] = {0, 0, 0};
  int c = 0;
  for (int j0 = 0; j0 < P.np; j0 += 32) {
    const int j = j0 + lane;
    bool hit = false;
    if (j < P.np && j != i) {
      // pair (lo, hi) with d = x_hi - x_lo as in addHertzian(lo, hi)
      const int lo = min(i, j), hi = max(i, j);
      const double* pl = pos + size_t(lo) * PS;
      const double* ph = pos + size_t(hi) * PS;
      double xdf = ph[0] - pl[0], ydf = ph[1] - pl[1], zdf = ph[2] - pl[2];
      xdf = xdf - double(g.nx * nint_d(xdf / g.nx));
      ydf = ydf - double(g.ny * nint_d(ydf / g.ny));
      zdf = zdf - double(g.nz * nint_d(zdf / g.nz));
      double rsq = xdf * xdf + ydf * ydf + zdf * zdf;
      if (nbr && rsq < nbr_pre) hit = sqrt(rsq) - 2.0 * P.rdim < gap_cut;
      if (rsq <= mxrsqcut) {
        double rrr = sqrt(rsq);
        double sgn = (i == lo) ? -1.0 : 1.0;
        if (rrr <= P.hz_rmin) {
          double ggg = (rrr <= P.hz_rcap) ? gmin : 5.0 * 0.5 * P.hz_k * pow(P.hz_rmin - rrr, 1.5);
          f[0] += sgn * (ggg * xdf / rrr);
          f[1] += sgn * (ggg * ydf / rrr);
          f[2] += sgn * (ggg * zdf / rrr);
        }
        if (P.lub && !P.closure && rrr <= rparcut) {
          double ux = xdf / rrr, uy = ydf / rrr, uz = zdf / rrr;
          if (rrr <= rparcap) rrr = rparcap;
          double dotuv = ux * (pl[3] - ph[3]) + uy * (pl[4] - ph[4]) + uz * (pl[5] - ph[5]);
          double cc = lubfactor * dotuv * (1.0 / (rrr - rpar) - 1.0);
          fl[0] += sgn * (cc * ux);
          fl[1] += sgn * (cc * uy);
          fl[2] += sgn * (cc * uz);
        }
      }
    }
    if (nbr) {
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      const int slot = c + __popc(m & ((1u << lane) - 1u));
      if (hit) {
        if (slot < NBCAP) nbr[size_t(i) * NBCAP + slot] = j;
        else raise_error(err, LBX_DEV_LIST_OVERFLOW, step, i);
      }
      c += __popc(m);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      f[d] += __shfl_down_sync(0xffffffffu, f[d], o);
      fl[d] += __shfl_down_sync(0xffffffffu, fl[d], o);
    }
  if (lane == 0) {
    for (int d = 0; d < 3; ++d) {
      acc[size_t(i) * AS + 6 + d] += f[d];
      acc[size_t(i) * AS + 12 + d] += fl[d];
    }
    if (nbr) cnt[i] = min(c, NBCAP);
  }
}

// ---------------------------------------------------------------------------
// learned closure in the step
// ---------------------------------------------------------------------------
__device__ __forceinline__ void min_image(const Geom& g, const double* pl, const double* ph, double d[3]) {
  d[0] = ph[0] - pl[0];
  d[1] = ph[1] - pl[1];
  d[2] = ph[2] - pl[2];
  d[0] = d[0] - double(g.nx * nint_d(d[0] / g.nx));
  d[1] = d[1] - double(g.ny * nint_d(d[1] / g.ny));
  d[2] = d[2] - double(g.nz * nint_d(d[2] / g.nz));
}

// one warp per close pair (i < j): the network inside its training envelope,
// the analytic squeeze force of addHertzian's lubrication branch outside it
__global__ void k_closure_pairs(PDev P, const double* __restrict__ pos, Geom g, const float* __restrict__ Wg,
                                int use_net, const int* __restrict__ nbr, const int* __restrict__ cnt, float* corr) {
  extern __shared__ float sm[];
  float* W = sm;
  float* bufs = W + MlpLayout::TOTAL;
  if (use_net) load_infer_weights(Wg, W);
  __syncthreads();
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  float* buf = bufs + warp * 2 * H;
  const int ntask = P.np * NBCAP;
  for (int t = blockIdx.x * nw + warp; t < ntask; t += gridDim.x * nw) {
    const int i = t / NBCAP, k = t % NBCAP;
    if (k >= cnt[i]) continue;
    const int j = nbr[size_t(i) * NBCAP + k];
    if (j < i) continue;
    const double* pi = pos + size_t(i) * PS;
    const double* pj = pos + size_t(j) * PS;
    // the network sees the pair where the templates sit (rounded centres)
    double d[3];
    {
      const int nn3[3] = {g.nx, g.ny, g.nz};
      for (int k = 0; k < 3; ++k) {
        double dk = double(nint_idx(pj[k], nn3[k]) - nint_idx(pi[k], nn3[k]));
        d[k] = dk - double(nn3[k]) * double(nint_d(dk / nn3[k]));
      }
    }
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double n[3] = {d[0] / r, d[1] / r, d[2] / r};
    double E[3][3], nc[3];
    const double sgn = lattice_frame(n, E, nc);
    const double dv[3] = {pj[3] - pi[3], pj[4] - pi[4], pj[5] - pi[5]};
    double oi[3] = {0, 0, 0}, oj[3] = {0, 0, 0};
    {
      double bi[3] = {pi[6], pi[7], pi[8]}, bj[3] = {pj[6], pj[7], pj[8]};
      to_lab(pi, bi, oi);
      to_lab(pj, bj, oj);
    }
    auto proj = [&](const double v[3], double f, double o[3]) {
      for (int a = 0; a < 3; ++a) o[a] = f * (v[0] * E[a][0] + v[1] * E[a][1] + v[2] * E[a][2]);
    };
    double fv[3], fi[3], fj[3];
    proj(dv, 1.0, fv);
    proj(oi, sgn, fi);
    proj(oj, sgn, fj);
    const double gapR = (r - 2.0 * P.rdim) / P.rdim;
    bool inside = use_net && gapR >= P.cl_gmin && gapR <= P.cl_gmax;
    for (int c = 0; c < 3 && inside; ++c)
      inside = fabs(fv[c]) <= P.cl_vmax && fabs(fi[c]) <= P.cl_vmax && fabs(fj[c]) <= P.cl_vmax;
    float out[12];
    for (int c = 0; c < 12; ++c) out[c] = 0.f;
    if (inside) {
      float x[DIN] = {float(gapR),  float(fv[0]), float(fv[1]),   float(fv[2]), float(fi[0]),
                      float(fi[1]), float(fi[2]), float(fj[0]),   float(fj[1]), float(fj[2]),
                      float(P.rdim), float(nc[1]), float(nc[2])};
      float y[DOUT];
      mlp_warp(W, x, y, buf);
      // forces back by E^T, torques (rows 3..5, 9..11) by det P * E^T
      for (int q = 0; q < 4; ++q) {
        const double f = (q & 1) ? sgn : 1.0;
        for (int c = 0; c < 3; ++c)
          out[3 * q + c] = float(f * (y[3 * q] * E[0][c] + y[3 * q + 1] * E[1][c] + y[3 * q + 2] * E[2][c]));
      }
    } else if (P.lub) {
      // the reference's lubrication on the centres themselves (addHertzian)
      double dc[3];
      min_image(g, pi, pj, dc);
      const double rc = sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
      const double nc[3] = {dc[0] / rc, dc[1] / rc, dc[2] / rc};
      const double rpar = 2.0 * P.rdim, rparcut = rpar + P.lub_rmin, rparcap = rpar + P.lub_rcap;
      if (rc <= rparcut) {
        const double lubfactor =
            P.lub_k * 6.0 * 3.141592653589793238462643383279502884 * pow(P.rdim * P.rdim, 2.0) / (rpar * rpar);
        double rr = rc <= rparcap ? rparcap : rc;
        double dotuv = nc[0] * (pi[3] - pj[3]) + nc[1] * (pi[4] - pj[4]) + nc[2] * (pi[5] - pj[5]);
        double cc = lubfactor * dotuv * (1.0 / (rr - rpar) - 1.0);
        for (int c = 0; c < 3; ++c) {
          out[c] = float(-cc * nc[c]);
          out[6 + c] = float(cc * nc[c]);
        }
      }
    }
    if (lane == 0)
      for (int c = 0; c < 12; ++c) corr[(size_t(i) * NBCAP + k) * 12 + c] = out[c];
  }
}

// per sphere, in ascending partner index: its share of every pair correction
__global__ void k_closure_accum(PDev P, const int* __restrict__ nbr, const int* __restrict__ cnt,
                                const float* __restrict__ corr, double* acc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
  for (int k = 0; k < cnt[i]; ++k) {
    const int j = nbr[size_t(i) * NBCAP + k];
    const float* cp;
    if (j > i) {
      cp = corr + (size_t(i) * NBCAP + k) * 12;
    } else {
      int kk = 0;
      while (kk < cnt[j] && nbr[size_t(j) * NBCAP + kk] != i) ++kk;
      if (kk >= cnt[j]) continue;
      cp = corr + (size_t(j) * NBCAP + kk) * 12 + 6;
    }
    for (int c = 0; c < 3; ++c) {
      F[c] += double(cp[c]);
      T[c] += double(cp[3 + c]);
    }
  }
  for (int c = 0; c < 3; ++c) {
    acc[size_t(i) * AS + 12 + c] += F[c];
    if (P.lrotate) acc[size_t(i) * AS + 9 + c] += T[c];
  }
}

// time_step_force_particles: force assembly f(t) = f_other + (f_bb(t+1/2) +
// f_bb(t-1/2))/2, leap-frog translation with the centred periodic image,
// the implicit mid-step quaternion update, then the accumulators restart
// from the external force and torque.
// the five records are distinct allocations (the two position and force
// slots and the accumulators): no store aliases a later load
__global__ void k_integrate(PDev P, const double* __restrict__ pos_cur, double* __restrict__ pos_next,
                            double* __restrict__ frc_cur, double* __restrict__ frc_next, double* __restrict__ acc,
                            Geom g, unsigned long long* err, int64_t step) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.np) return;
  const double* pc = pos_cur + size_t(a) * PS;
  double* pn = pos_next + size_t(a) * PS;
  double* fc = frc_cur + size_t(a) * FS;
  double* fo = frc_next + size_t(a) * FS;  // the slot of the previous step
  double* A = acc + size_t(a) * AS;
  for (int d = 0; d < 3; ++d) {
    fc[d] = A[6 + d] + A[12 + d];
    fc[3 + d] = A[d];
    fc[d] = fc[d] + (fc[3 + d] + fo[3 + d]) * 0.5;
  }
  if (P.lrotate)
    for (int d = 0; d < 3; ++d) {
      fc[6 + d] = A[9 + d];
      fc[9 + d] = A[3 + d];
      fc[6 + d] = fc[6 + d] + (fc[9 + d] + fo[9 + d]) * 0.5;
    }
  // nve_lf
  const double rmass = P.rmass;
  if (!P.kinematic && (fabs(fc[0]) * rmass > 0.5 || fabs(fc[1]) * rmass > 0.5 || fabs(fc[2]) * rmass > 0.5))
    raise_error(err, LBX_DEV_BIG_FORCE, step, a);
  double bv[3];
  for (int d = 0; d < 3; ++d) bv[d] = P.kinematic ? pc[3 + d] : pc[3 + d] + rmass * fc[d];
  double vm = sqrt(bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2]);
  if (!P.kinematic && vm > P.max_vel) raise_error(err, LBX_DEV_EXTREME_VEL, step, a);
  const int nn[3] = {g.nx, g.ny, g.nz};
  double xn[3];
  for (int d = 0; d < 3; ++d) {
    double cc = double(nn[d] + 1) * 0.5;
    double xs = (pc[d] + bv[d]) - cc;
    xn[d] = xs - double(nn[d]) * double(nint_d((1.0 / nn[d]) * xs)) + cc;
    if (xn[d] < 0.5 || xn[d] > double(nn[d]) + 0.5) raise_error(err, LBX_DEV_POSITION, step, a);
  }
  if (P.lrotate) {  // rot_midstep_impl_lf
    const double mass = 1.0 / rmass;
    const double rotin = 2.0 / 5.0 * mass * P.rdim * P.rdim;
    double oxx = pc[6], oyy = pc[7], ozz = pc[8];
    double q0 = pc[9], q1 = pc[10], q2 = pc[11], q3 = pc[12];
    double tqx = fc[6], tqy = fc[7], tqz = fc[8];
    double m[9];
    m[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
    m[1] = 2.0 * (q1 * q2 - q0 * q3);
    m[2] = 2.0 * (q1 * q3 + q0 * q2);
    m[3] = 2.0 * (q1 * q2 + q0 * q3);
    m[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
    m[5] = 2.0 * (q2 * q3 - q0 * q1);
    m[6] = 2.0 * (q1 * q3 - q0 * q2);
    m[7] = 2.0 * (q2 * q3 + q0 * q1);
    m[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
    double opx = oxx, opy = oyy, opz = ozz;
    double delx = (tqx * m[0] + tqy * m[3] + tqz * m[6]) / rotin + (rotin - rotin) * opy * opz / rotin;
    double dely = (tqx * m[1] + tqy * m[4] + tqz * m[7]) / rotin + (rotin - rotin) * opz * opx / rotin;
    double delz = (tqx * m[2] + tqy * m[5] + tqz * m[8]) / rotin + (rotin - rotin) * opx * opy / rotin;
    opx = oxx + delx * 0.5;
    opy = oyy + dely * 0.5;
    opz = ozz + delz * 0.5;
    double dq0 = (-q1 * opx - q2 * opy - q3 * opz) * 0.5;
    double dq1 = (q0 * opx - q3 * opy + q2 * opz) * 0.5;
    double dq2 = (q3 * opx + q0 * opy - q1 * opz) * 0.5;
    double dq3 = (-q2 * opx + q1 * opy + q0 * opz) * 0.5;
    double qn0 = q0 + dq0 * 0.5, qn1 = q1 + dq1 * 0.5, qn2 = q2 + dq2 * 0.5, qn3 = q3 + dq3 * 0.5;
    double rn = 1.0 / sqrt(qn0 * qn0 + qn1 * qn1 + qn2 * qn2 + qn3 * qn3);
    qn0 *= rn; qn1 *= rn; qn2 *= rn; qn3 *= rn;
    oxx += delx; oyy += dely; ozz += delz;
    pn[6] = oxx; pn[7] = oyy; pn[8] = ozz;
    opx = oxx; opy = oyy; opz = ozz;
    int itq = 0;
    double eps = 1.0e9;
    while (itq < 20 && eps > 1.0e-24) {  // at most 20 fixed-point iterations
      ++itq;
      dq0 = (-qn1 * opx - qn2 * opy - qn3 * opz) * 0.5;
      dq1 = (qn0 * opx - qn3 * opy + qn2 * opz) * 0.5;
      dq2 = (qn3 * opx + qn0 * opy - qn1 * opz) * 0.5;
      dq3 = (-qn2 * opx + qn1 * opy + qn0 * opz) * 0.5;
      double a0 = qn0 + dq0 * 0.5, a1 = qn1 + dq1 * 0.5, a2 = qn2 + dq2 * 0.5, a3 = qn3 + dq3 * 0.5;
      rn = 1.0 / sqrt(a0 * a0 + a1 * a1 + a2 * a2 + a3 * a3);
      a0 *= rn; a1 *= rn; a2 *= rn; a3 *= rn;
      eps = (a0 - qn0) * (a0 - qn0) + (a1 - qn1) * (a1 - qn1) + (a2 - qn2) * (a2 - qn2) + (a3 - qn3) * (a3 - qn3);
      qn0 = a0; qn1 = a1; qn2 = a2; qn3 = a3;
    }
    q0 += dq0; q1 += dq1; q2 += dq2; q3 += dq3;
    rn = 1.0 / sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    pn[9] = q0 * rn; pn[10] = q1 * rn; pn[11] = q2 * rn; pn[12] = q3 * rn;
  } else {
    for (int k = 6; k < PS; ++k) pn[k] = pc[k];
  }
  for (int d = 0; d < 3; ++d) { pn[d] = xn[d]; pn[3 + d] = bv[d]; }
  if (P.kinematic)  // prescribed motion: the centre moves with the set velocity, v / omega / q are kept
    for (int k = 3; k < PS; ++k) pn[k] = pc[k];
  if (P.kinematic == 2)  // frozen geometry: the centre stays, the wall still moves with v and omega
    for (int d = 0; d < 3; ++d) pn[d] = pc[d];
  for (int d = 0; d < 3; ++d) {
    fo[d] = P.ext_f[d];
    fo[3 + d] = 0;
    A[d] = 0;             // f_bb
    A[6 + d] = P.ext_f[d];  // f_other restarts at the external force
    A[12 + d] = 0;
    if (P.lrotate) {
      fo[6 + d] = P.ext_t[d];
      fo[9 + d] = 0;
      A[3 + d] = 0;
      A[9 + d] = P.ext_t[d];
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PDev pdev(const Ctx& c) {
  const ParticleState& s = *c.part;
  PDev d;
  d.np = s.np;
  d.rmax = s.rmax;
  d.sphereMax = s.sphereMax;
  d.tw = s.tw;
  d.lrotate = s.lrotate;
  d.rdim = s.rdim;
  d.rmass = double(c.p.rmass);
  d.max_vel = double(c.p.max_vel);
  d.tmpl = s.tmpl;
  d.offs = s.offs;
  d.offs_bb = s.offs ? s.offs + s.n_solid : nullptr;
  d.n_surf = s.n_surf;
  d.n_solid = s.n_solid;
  d.n_bb = s.n_bb;
  d.offs_shell = s.offs ? s.offs + s.n_solid + s.n_bb : nullptr;
  d.n_shell = s.n_shell;
  d.shell_r2 = s.shell_r2;
  d.owner = s.owner;
  d.bin_cnt = s.bin_cnt;
  d.bin_list = s.bin_list;
  d.nbx = s.nbx;
  d.nby = s.nby;
  d.nbz = s.nbz;
  for (int k = 0; k < 3; ++k) {
    d.ext_f[k] = double(c.p.ext_force[k]);
    d.ext_t[k] = double(c.p.ext_torque[k]);
  }
  d.hz_k = double(c.p.hz_k);
  d.hz_rmin = double(c.p.hz_rmin);
  d.hz_rcap = double(c.p.hz_rcap);
  d.lub = c.p.lubrication;
  d.lub_k = double(c.p.lubric_k);
  d.lub_rmin = double(c.p.lubric_rmin);
  d.lub_rcap = double(c.p.lubric_rcap);
  d.kinematic = c.p.kinematic;
  d.closure = c.p.closure;
  d.cl_gmin = c.p.closure_gap_min;
  d.cl_gmax = c.p.closure_gap_max;
  d.cl_vmax = c.p.closure_vmax;
  d.exact_tiles = c.p.exact_tiles;
  d.crowd = s.crowd;
  return d;
}

// spherical_template (main.CUF:1990-2130), in FP64 (rdim^2 and the integer
// squared distances are exact in either precision)
static std::vector<int8_t> make_template(double rdim, int& rmin, int& rmax) {
  const double sqrcut = rdim * rdim;
  rmin = int(std::floor(rdim));
  rmax = int(rdim + 1.0);
  const int w = 2 * rmax + 1;
  std::vector<int8_t> t(size_t(w) * w * w, LBX_FLUID_FLUID);
  auto at3 = [&](int i, int j, int k) -> int8_t& { return t[(i + rmax) + w * ((j + rmax) + w * (k + rmax))]; };
  for (int k = -rmax; k <= rmax; ++k)
    for (int j = -rmax; j <= rmax; ++j)
      for (int i = -rmax; i <= rmax; ++i)
        if (double(i * i + j * j + k * k) <= sqrcut) at3(i, j, k) = LBX_FLUID_SPHEREDEAD;
  for (int k = -rmin; k <= rmin; ++k)
    for (int j = -rmin; j <= rmin; ++j)
      for (int i = -rmin; i <= rmin; ++i)
        if (at3(i, j, k) == LBX_FLUID_SPHEREDEAD)
          for (int l = 1; l < Q; ++l)
            if (at3(i + ex(l), j + ey(l), k + ez(l)) == LBX_FLUID_FLUID) {
              at3(i, j, k) = LBX_FLUID_SPHERELIST;
              break;
            }
  at3(0, 0, 0) = LBX_FLUID_PARTICLECM;
  return t;
}

int particles_create(Ctx& c) {
  if (c.ncomp != 2) return LBX_ERR_STATE;
  if (c.nx % TILEX || c.ny % TILEY || c.nz % TILEZ) return LBX_ERR_ARG;  // reference tile grid
  ParticleState* s = new ParticleState();
  c.part = s;
  int cap = c.p.max_particles;
  s->rdim = double(c.p.radius);
  int rmin;
  std::vector<int8_t> t = make_template(s->rdim, rmin, s->rmax);
  s->tw = 2 * s->rmax + 1;
  s->sphereMax = s->rmax * s->rmax;
  if (c.nx < 2 * s->rmax + 2 || c.ny < 2 * s->rmax + 2 || c.nz < 2 * s->rmax + 2) return LBX_ERR_ARG;
  s->lrotate = c.p.lrotate ? 1 : 0;
  s->nbx = (c.nx + BINW - 1) / BINW;
  s->nby = (c.ny + BINW - 1) / BINW;
  s->nbz = (c.nz + BINW - 1) / BINW;
  size_t nbins = size_t(s->nbx) * s->nby * s->nbz;
  auto ok = [](cudaError_t e) { return e == cudaSuccess; };
  for (int k = 0; k < 2; ++k) {
    if (!ok(cudaMalloc(&s->pos[k], size_t(cap) * PS * 8))) return LBX_ERR_ALLOC;
    if (!ok(cudaMalloc(&s->frc[k], size_t(cap) * FS * 8))) return LBX_ERR_ALLOC;
    cudaMemsetAsync(s->pos[k], 0, size_t(cap) * PS * 8, c.stream);
    cudaMemsetAsync(s->frc[k], 0, size_t(cap) * FS * 8, c.stream);
  }
  if (!ok(cudaMalloc(&s->acc, size_t(cap) * AS * 8))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->tmpl, t.size()))) return LBX_ERR_ALLOC;
  // offset lists: solid template cells (surface first), then the bounce-back
  // list (surface cells, then the rest of the reach d^2 < sphereMax)
  std::vector<int> offs;
  const int R = s->rmax, w = s->tw;
  auto tv = [&](int i, int j, int k) { return int(t[(i + R) + w * ((j + R) + w * (k + R))]); };
  for (int pass = 0; pass < 3; ++pass)
    for (int k = -R; k <= R; ++k)
      for (int j = -R; j <= R; ++j)
        for (int i = -R; i <= R; ++i) {
          const int v = tv(i, j, k);
          const bool take = pass == 0 ? v == LBX_FLUID_SPHERELIST
                                      : pass == 1 ? v == LBX_FLUID_SPHEREDEAD : v == LBX_FLUID_PARTICLECM;
          if (take) offs.push_back(pack_off(i, j, k, v));
        }
  s->n_solid = int(offs.size());
  for (int q = 0; q < s->n_solid; ++q)
    if (((offs[size_t(q)] >> 24) & 255) == LBX_FLUID_SPHERELIST) s->n_surf = q + 1;
  for (int q = 0; q < s->n_surf; ++q) offs.push_back(offs[size_t(q)]);
  for (int k = -R; k <= R; ++k)
    for (int j = -R; j <= R; ++j)
      for (int i = -R; i <= R; ++i)
        if (i * i + j * j + k * k < s->sphereMax && tv(i, j, k) != LBX_FLUID_SPHERELIST)
          offs.push_back(pack_off(i, j, k, tv(i, j, k)));
  s->n_bb = int(offs.size()) - s->n_solid;
  // density shell: the template's fluid belt (every offset outside the
  // template with a D3Q27 neighbour inside it; all lie within rdim + sqrt 3 of
  // the centre), then the template cells with their values (solid template
  // cells are fluid only when the tile-list coverage left them out, so they
  // are tested before pulling)
  const double rs = s->rdim + std::sqrt(3.0);
  s->shell_r2 = int(std::floor(rs * rs));
  const int RS = int(std::ceil(rs));
  if (RS > 60) return LBX_ERR_ARG;  // offsets are packed in 8 bits
  auto solid = [&](int i, int j, int k) {
    return std::abs(i) <= R && std::abs(j) <= R && std::abs(k) <= R && tv(i, j, k) != LBX_FLUID_FLUID;
  };
  for (int k = -RS; k <= RS; ++k)
    for (int j = -RS; j <= RS; ++j)
      for (int i = -RS; i <= RS; ++i) {
        if (solid(i, j, k)) continue;
        bool belt = false;
        for (int e = 1; e < Q27 && !belt; ++e) belt = solid(i + ex27(e), j + ey27(e), k + ez27(e));
        if (belt) offs.push_back(pack_off(i, j, k, LBX_FLUID_FLUID));
      }
  for (int k = -R; k <= R; ++k)
    for (int j = -R; j <= R; ++j)
      for (int i = -R; i <= R; ++i)
        if (solid(i, j, k)) offs.push_back(pack_off(i, j, k, tv(i, j, k)));
  s->n_shell = int(offs.size()) - s->n_solid - s->n_bb;
  if (!ok(cudaMalloc(&s->offs, offs.size() * 4))) return LBX_ERR_ALLOC;
  cudaMemcpyAsync(s->offs, offs.data(), offs.size() * 4, cudaMemcpyHostToDevice, c.stream);
  if (!ok(cudaMalloc(&s->owner, size_t(c.n) * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->bin_cnt, nbins * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->bin_list, nbins * BIN_CAP * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->wclosure, size_t(LBX_CLOSURE_NWEIGHTS) * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->nbr, size_t(cap) * NBCAP * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->nbr_cnt, size_t(cap) * 4))) return LBX_ERR_ALLOC;
  if (!ok(cudaMalloc(&s->crowd, size_t(cap)))) return LBX_ERR_ALLOC;
  if (!ok(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking)) ||
      !ok(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming)) ||
      !ok(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming)) ||
      !ok(cudaEventCreateWithFlags(&s->ev_flags, cudaEventDisableTiming)) ||
      !ok(cudaEventCreateWithFlags(&s->ev_owner, cudaEventDisableTiming)))
    return LBX_ERR_CUDA;
  if (!ok(cudaMalloc(&s->corr, size_t(cap) * NBCAP * 12 * 4))) return LBX_ERR_ALLOC;
  cudaMemsetAsync(s->acc, 0, size_t(cap) * AS * 8, c.stream);
  cudaMemsetAsync(s->owner, 0xFF, size_t(c.n) * 4, c.stream);
  cudaMemcpyAsync(s->tmpl, t.data(), t.size(), cudaMemcpyHostToDevice, c.stream);
  cudaStreamSynchronize(c.stream);
  return launch_status();
}

void particles_destroy(Ctx& c) {
  ParticleState* s = c.part;
  if (!s) return;
  for (int k = 0; k < 2; ++k) {
    if (s->pos[k]) cudaFree(s->pos[k]);
    if (s->frc[k]) cudaFree(s->frc[k]);
  }
  if (s->acc) cudaFree(s->acc);
  if (s->tmpl) cudaFree(s->tmpl);
  if (s->offs) cudaFree(s->offs);
  if (s->owner) cudaFree(s->owner);
  if (s->bin_cnt) cudaFree(s->bin_cnt);
  if (s->bin_list) cudaFree(s->bin_list);
  if (s->wclosure) cudaFree(s->wclosure);
  if (s->nbr) cudaFree(s->nbr);
  if (s->nbr_cnt) cudaFree(s->nbr_cnt);
  if (s->crowd) cudaFree(s->crowd);
  if (s->corr) cudaFree(s->corr);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->ev_flags) cudaEventDestroy(s->ev_flags);
  if (s->ev_owner) cudaEventDestroy(s->ev_owner);
  if (s->aux) cudaStreamDestroy(s->aux);
  delete s;
  c.part = nullptr;
}

static int rebuild_bins(Ctx& c, const double* pos, cudaStream_t st) {
  ParticleState& s = *c.part;
  PDev P = pdev(c);
  Geom g = geom(c);
  size_t nbins = size_t(s.nbx) * s.nby * s.nbz;
  cudaMemsetAsync(s.bin_cnt, 0, nbins * 4, st);
  k_bins<<<(s.np * 32 + 255) / 256, 256, 0, st>>>(P, pos, g, c.d_err, c.step + 1);
  k_bins_sort<<<int((nbins + 255) / 256), 256, 0, st>>>(P, int(nbins));
  k_crowd<<<(s.np * 32 + 255) / 256, 256, 0, st>>>(P, pos, g);
  return launch_status();
}

// flags and owners of the spheres at `pos` (every other cell fluid, no owner)
//   prev: positions of the last stamping of the owners (nullptr: clear the
//   whole owner and flag arrays).  Otherwise `flags` must already be all
//   fluid, which the end of the step before guarantees (k_unstamp).
static int compute_flags(Ctx& c, const double* pos, int8_t* flags, const double* prev) {
  ParticleState& s = *c.part;
  PDev P = pdev(c);
  Geom g = geom(c);
  if (prev) {
    if (!s.owner_clear) k_unstamp<<<s.np, 256, 0, c.stream>>>(P, prev, g, nullptr, s.owner);
  } else {
    cudaMemsetAsync(flags, LBX_FLUID_FLUID, size_t(c.n), c.stream);
    cudaMemsetAsync(s.owner, 0xFF, size_t(c.n) * 4, c.stream);
  }
  s.owner_clear = 0;
  k_stamp<<<s.np, 256, 0, c.stream>>>(P, pos, g);
  k_stamp_flags<<<s.np, 256, 0, c.stream>>>(P, pos, g, flags);
  return launch_status();
}

// set_particles: the state read_input_atom builds (main.CUF:1230-1350) and
// the step-0 flags of setupRho_Pops (main.CUF:2586-2600).
int particles_set(Ctx& c, int n, const double* h_x, const double* h_v, const double* h_om, const double* h_q) {
  ParticleState* s = c.part;
  if (!s || n < 1 || n > c.p.max_particles) return LBX_ERR_ARG;
  s->np = n;
  std::vector<double> pos(size_t(n) * PS, 0.0), frc(size_t(n) * FS, 0.0);
  for (int a = 0; a < n; ++a) {
    for (int d = 0; d < 3; ++d) {
      pos[size_t(a) * PS + d] = h_x[3 * a + d];
      pos[size_t(a) * PS + 3 + d] = h_v ? h_v[3 * a + d] : 0.0;
      pos[size_t(a) * PS + 6 + d] = h_om ? h_om[3 * a + d] : 0.0;
      frc[size_t(a) * FS + d] = double(c.p.ext_force[d]);
      if (c.p.lrotate) frc[size_t(a) * FS + 6 + d] = double(c.p.ext_torque[d]);
    }
    for (int k = 0; k < 4; ++k) pos[size_t(a) * PS + 9 + k] = h_q ? h_q[4 * a + k] : (k == 0 ? 1.0 : 0.0);
  }
  for (int k = 0; k < 2; ++k) {
    cudaMemcpyAsync(s->pos[k], pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, c.stream);
    cudaMemcpyAsync(s->frc[k], frc.data(), frc.size() * 8, cudaMemcpyHostToDevice, c.stream);
  }
  // the FP64 accumulators start at zero (the first step has no external force
  // in its total, as in the reference, whose myf2_d is first set at the end
  // of step 1)
  cudaMemsetAsync(s->acc, 0, size_t(c.p.max_particles) * AS * 8, c.stream);
  s->pcur = 0;
  s->active = 1;
  // step-0 flags into the slot the first step will recompute; the slot the
  // first step treats as "previous" stays all fluid, as in the reference
  int slot = 1 - c.fcur;
  int rc = rebuild_bins(c, s->pos[0], c.stream);
  if (rc) return rc;
  // both flag slots all fluid (the step-0 flags go into `slot`)
  cudaMemsetAsync(c.flags[1 - slot], LBX_FLUID_FLUID, size_t(c.n), c.stream);
  rc = compute_flags(c, s->pos[0], c.flags[slot], nullptr);
  s->flags_last = slot;
  if (!rc) rc = cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : LBX_ERR_CUDA;
  return rc;
}

// One step with particles, main.CUF:130-241, as the stages the reference
// launches (each a kernel-level entry point of the C ABI as well):
//   pre:   lists, flags, drain, densities, fill, wetting
//   fluid: the colour-gradient step with flags
//   post:  bounce-back (n2p, copy, wall), pair forces (+ closure), integrator
//          and the buffer swap
// particles_pre / particles_post group them so that an ensemble can put the
// fluid kernels of all its boxes into one launch.
namespace {
struct Stage {  // the buffers and constants every stage launch needs
  ParticleState& s;
  Geom g;
  PDev P;
  int fo, fn;
  const double* pc;
  const double* po;
  int64_t st;
  explicit Stage(Ctx& c)
      : s(*c.part), g(geom(c)), P(pdev(c)), fo(c.fcur), fn(1 - c.fcur), pc(c.part->pos[c.part->pcur]),
        po(c.part->pos[1 - c.part->pcur]), st(c.step + 1) {}
};
}  // namespace

static int lists_on(Ctx& c, cudaStream_t st) {
  Stage t(c);
  return rebuild_bins(c, t.pc, st);
}

int part_lists(Ctx& c) { return lists_on(c, c.stream); }

int part_flags(Ctx& c) {
  Stage t(c);
  return compute_flags(c, t.pc, c.flags[t.fn], t.po);
}

static int drain_on(Ctx& c, cudaStream_t st) {
  Stage t(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    k_drain<S><<<t.s.np, 256, 0, st>>>(t.P, t.pc, t.po, t.s.acc, (const S*)c.pops[c.cur],
                                              (const S*)c.pops[1 - c.cur], t.g, make_shift<C>(c), c.flags[t.fo],
                                              c.flags[t.fn], (const C*)c.rho[0], (const C*)c.rho[1]);
    return launch_status();
  });
}

int part_drain(Ctx& c) { return drain_on(c, c.stream); }

// init_rho*_CG with flags: every cell (two-pass schedule) or only the fluid
// cells the particle kernels read (single-pass schedule, whose fluid kernel
// pulls its own densities)
int part_rho(Ctx& c) {
  Stage t(c);
  LaunchDims d = cell_dims(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    const S* A = (const S*)c.pops[c.cur];
    S* B = (S*)c.pops[1 - c.cur];
    if (c.fused != 2)
      k_rho_p<S><<<d.grid, d.block, 0, c.stream>>>(A, B, t.g, make_shift<C>(c), c.flags[t.fo], c.flags[t.fn],
                                                   (C*)c.phi, (C*)c.rho[0], (C*)c.rho[1], c.d_err, t.st);
    else
      k_rho_shell<S><<<t.s.np, 256, 0, c.stream>>>(t.P, t.pc, t.po, A, t.g, make_shift<C>(c), c.flags[t.fo],
                                                    c.flags[t.fn], (C*)c.rho[0], (C*)c.rho[1]);
    return launch_status();
  });
}

int part_fill(Ctx& c) {
  Stage t(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    k_fill<S><<<t.s.np, 256, 0, c.stream>>>(t.P, t.pc, t.po, t.s.acc, (const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur],
                                             c.fused == 2 ? (S*)c.pops[c.cur] : nullptr, t.g, make_shift<C>(c),
                                             make_lattice<C>(), c.flags[t.fo], c.flags[t.fn], (C*)c.rho[0],
                                             (C*)c.rho[1], (C*)c.phi);
    return launch_status();
  });
}

int part_virtual(Ctx& c) {
  Stage t(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    k_virtual<S><<<t.s.np, 256, 0, c.stream>>>(t.P, t.pc, t.g, c.p.wetting == LBX_WET_NEUTRAL ? 1 : 0,
                                                (const S*)c.pops[c.cur], make_shift<C>(c), c.flags[t.fo],
                                                c.flags[t.fn], (C*)c.rho[0], (C*)c.rho[1], (C*)c.phi,
                                                make_lattice<C>());
    return launch_status();
  });
}

// With the single-pass schedule the stages that do not feed the next one run
// on the second stream: the particle lists (read by the bounce-back only)
// beside the flags, and the drain (it reads the densities of the cells the
// spheres now cover, which the density shell does not write) beside the
// density shell.  The fill adds to the same accumulators as the drain, after
// it, and the fluid kernel's flags wait for nothing else: the join is before
// the fill.  The two-pass schedule's density pass writes every cell, so it
// keeps the reference's order on one stream.  forks = false: every stage on
// the context's stream (an ensemble, whose boxes already run side by side on
// their own streams: a second stream per box measured slower there, 1.65
// against 1.38 ms per step with 48 boxes).
int particles_pre(Ctx& c, bool forks) {
  ParticleState& s = *c.part;
  // without forks the step's end clears no owners, and a graph captured
  // from these stages replays them unchanged: clear them here every time
  // (again, if a step with forks already did; clearing is idempotent)
  if (!forks) s.owner_clear = 0;
  if (c.fused != 2 || !forks) {
    int rc = part_lists(c);
    if (!rc) rc = part_flags(c);
    if (!rc) rc = part_drain(c);
    if (!rc) rc = part_rho(c);
    if (!rc) rc = part_fill(c);
    if (!rc) rc = part_virtual(c);
    return rc;
  }
  if (cudaEventRecord(s.ev_fork, c.stream) != cudaSuccess || cudaStreamWaitEvent(s.aux, s.ev_fork, 0) != cudaSuccess)
    return LBX_ERR_CUDA;
  int rc = lists_on(c, s.aux);
  if (!rc) rc = part_flags(c);
  if (!rc && (cudaEventRecord(s.ev_flags, c.stream) != cudaSuccess ||
              cudaStreamWaitEvent(s.aux, s.ev_flags, 0) != cudaSuccess))
    rc = LBX_ERR_CUDA;
  if (!rc) rc = drain_on(c, s.aux);
  if (!rc && cudaEventRecord(s.ev_join, s.aux) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc) rc = part_rho(c);
  if (!rc && cudaStreamWaitEvent(c.stream, s.ev_join, 0) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc) rc = part_fill(c);
  if (!rc) rc = part_virtual(c);
  return rc;
}

int particles_fluid(Ctx& c) {
  const int fo = c.fcur, fn = 1 - c.fcur;
  if (c.fused == 2) return fluid_lean_particles(c, fo, fn);
  Geom g = geom(c);
  LaunchDims d = cell_dims(c);
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    kt_begin(c);
    if (c.p.model == LBX_MODEL_CG_DIFFDENS)
      k_collide_p<S, true><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], g,
                                                             make_shift<C>(c), (const C*)c.phi, (const C*)c.rho[0],
                                                             (const C*)c.rho[1], c.flags[fo], c.flags[fn],
                                                             make_cg<C>(c));
    else
      k_collide_p<S, false><<<d.grid, d.block, 0, c.stream>>>((const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], g,
                                                              make_shift<C>(c), (const C*)c.phi, (const C*)c.rho[0],
                                                              (const C*)c.rho[1], c.flags[fo], c.flags[fn],
                                                              make_cg<C>(c));
    kt_end(c);
    return launch_status();
  });
}

// partBB_CG (BB_N2P), partBB_CG_p2n (BB_COPY), partBB_CG_p2n2 (BB_WALL)
int part_bb(Ctx& c, int mode) {
  Stage t(c);
  if (mode < 1 || mode > BB_ALL) return LBX_ERR_ARG;
  return by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    k_bb<S><<<t.s.np, 256, 0, c.stream>>>(t.P, t.pc, t.s.acc, (S*)c.pops[1 - c.cur], t.g, make_shift<C>(c),
                                           make_lattice<C>(), c.flags[t.fn], (const C*)c.rho[0], (const C*)c.rho[1],
                                           mode);
    return launch_status();
  });
}

// inter_force_particles: Hertz and analytic lubrication, then the closure
static int pairs_on(Ctx& c, cudaStream_t st) {
  Stage t(c);
  ParticleState& s = t.s;
  const int warp_blocks = (s.np * 32 + 255) / 256;
  // with the closure, the same all-pairs pass lists each sphere's close
  // partners; the network's gap is that of the rounded centres, up to
  // sqrt 3 closer than the centres' own
  const double cut = c.p.closure ? fmax(double(c.p.closure_gap_max) * s.rdim + 1.75,
                                        c.p.lubrication ? double(c.p.lubric_rmin) : 0.0)
                                 : 0.0;
  k_pairs<<<warp_blocks, 256, 0, st>>>(t.P, t.pc, s.acc, t.g, cut, c.p.closure ? s.nbr : nullptr, s.nbr_cnt,
                                        c.d_err, t.st);
  if (c.p.closure) {
    const int use_net = s.closure_ready;
    size_t smem = sizeof(float) * (size_t(LBX_CLOSURE_NWEIGHTS) + 8 * 2 * H);
    int blocks = (s.np * NBCAP + 7) / 8;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_closure_pairs<<<blocks, 256, smem, st>>>(t.P, t.pc, t.g, s.wclosure, use_net, s.nbr, s.nbr_cnt, s.corr);
    k_closure_accum<<<(s.np + 127) / 128, 128, 0, st>>>(t.P, s.nbr, s.nbr_cnt, s.corr, s.acc);
  }
  return launch_status();
}

int part_pairs(Ctx& c) { return pairs_on(c, c.stream); }

// the previous step's flags (stamped at the previous positions) are not read
// again: clear them, so that the next step stamps into a fluid slot
static int unstamp_on(Ctx& c, cudaStream_t st) {
  Stage t(c);
  k_unstamp<<<t.s.np, 256, 0, st>>>(t.P, t.po, t.g, c.flags[t.fo], nullptr);
  return launch_status();
}

// time_step_force_particles, then the end of the step: every ping-pong
// index (populations, flags, particle records) flips
static int integrate_flip(Ctx& c) {
  Stage t(c);
  ParticleState& s = t.s;
  k_integrate<<<(s.np + 127) / 128, 128, 0, c.stream>>>(t.P, t.pc, s.pos[1 - s.pcur], s.frc[s.pcur],
                                                        s.frc[1 - s.pcur], s.acc, t.g, c.d_err, t.st);
  int rc = launch_status();
  if (rc) return rc;
  c.cur = 1 - c.cur;
  c.fcur = t.fn;
  s.flags_last = t.fn;
  s.pcur = 1 - s.pcur;
  c.step += 1;
  return 0;
}

int part_integrate(Ctx& c) {
  int rc = unstamp_on(c, c.stream);
  return rc ? rc : integrate_flip(c);
}

// The bounce-back on the context's stream; beside it, on the second stream,
// the pair forces (accumulators of their own, acc[6..14], against acc[0..5]
// of the bounce-back) and the clearing of the previous step's flags (the
// bounce-back reads this step's); both join before the integrator, which
// overwrites the previous positions the clearing reads.  After the
// bounce-back, the last reader of the owners, the second stream clears them
// at this step's positions beside the integrator (which writes the next
// positions, not these), joined at the end of the step; the next flag stage
// then stamps without clearing first.  forks = false: one stream, as in
// particles_pre.
int particles_post(Ctx& c, bool forks) {
  ParticleState& s = *c.part;
  if (!forks) {
    int rc = pairs_on(c, c.stream);
    if (!rc) rc = unstamp_on(c, c.stream);
    if (!rc) rc = part_bb(c, BB_ALL);
    if (!rc) rc = integrate_flip(c);
    return rc;
  }
  if (cudaEventRecord(s.ev_fork, c.stream) != cudaSuccess || cudaStreamWaitEvent(s.aux, s.ev_fork, 0) != cudaSuccess)
    return LBX_ERR_CUDA;
  int rc = pairs_on(c, s.aux);
  if (!rc) rc = unstamp_on(c, s.aux);
  if (!rc && cudaEventRecord(s.ev_join, s.aux) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc) rc = part_bb(c, BB_ALL);
  if (!rc && (cudaEventRecord(s.ev_flags, c.stream) != cudaSuccess ||
              cudaStreamWaitEvent(s.aux, s.ev_flags, 0) != cudaSuccess))
    rc = LBX_ERR_CUDA;
  if (!rc) {
    Stage t(c);
    k_unstamp<<<s.np, 256, 0, s.aux>>>(t.P, t.pc, t.g, nullptr, s.owner);
    rc = launch_status();
  }
  if (!rc && cudaEventRecord(s.ev_owner, s.aux) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc && cudaStreamWaitEvent(c.stream, s.ev_join, 0) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc) rc = integrate_flip(c);
  if (!rc && cudaStreamWaitEvent(c.stream, s.ev_owner, 0) != cudaSuccess) rc = LBX_ERR_CUDA;
  if (!rc) s.owner_clear = 1;
  return rc;
}

int particles_step(Ctx& c) {
  int rc = particles_pre(c, true);
  if (!rc) rc = particles_fluid(c);
  if (!rc) rc = particles_post(c, true);
  return rc;
}

int particles_get(Ctx& c, double* x, double* v, double* om, double* q, double* f, double* t) {
  ParticleState* s = c.part;
  if (!s || !s->active) return LBX_ERR_STATE;
  int n = s->np;
  std::vector<double> pos(size_t(n) * PS), frc(size_t(n) * FS);
  cudaMemcpyAsync(pos.data(), s->pos[s->pcur], pos.size() * 8, cudaMemcpyDeviceToHost, c.stream);
  // total force / torque the integrator used in the last step
  cudaMemcpyAsync(frc.data(), s->frc[1 - s->pcur], frc.size() * 8, cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) return LBX_ERR_CUDA;
  for (int a = 0; a < n; ++a) {
    for (int d = 0; d < 3; ++d) {
      if (x) x[3 * a + d] = pos[size_t(a) * PS + d];
      if (v) v[3 * a + d] = pos[size_t(a) * PS + 3 + d];
      if (om) om[3 * a + d] = pos[size_t(a) * PS + 6 + d];
      if (f) f[3 * a + d] = frc[size_t(a) * FS + d];
      if (t) t[3 * a + d] = frc[size_t(a) * FS + 6 + d];
    }
    if (q)
      for (int k = 0; k < 4; ++k) q[4 * a + k] = pos[size_t(a) * PS + 9 + k];
  }
  return 0;
}

int particles_set_closure(Ctx& c, const float* h_w) {
  ParticleState* s = c.part;
  if (!s) return LBX_ERR_STATE;
  if (cudaMemcpyAsync(s->wclosure, h_w, size_t(LBX_CLOSURE_NWEIGHTS) * 4, cudaMemcpyHostToDevice, c.stream) !=
      cudaSuccess)
    return LBX_ERR_CUDA;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_closure_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(sizeof(float) * (size_t(LBX_CLOSURE_NWEIGHTS) + 8 * 2 * H)));
    attr = true;
  }
  s->closure_ready = 1;
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : LBX_ERR_CUDA;
}

// The bounce-back links of the flags lbx_get_flags reports (those of the last
// step, or of lbx_set_particles before the first step) at the positions that
// stamped them; sorted by (sphere, cell, direction).
int particles_links(Ctx& c, int32_t* h_cell, int8_t* h_dir, int32_t* h_sph, int64_t cap, int64_t* h_n) {
  ParticleState* s = c.part;
  if (!s || !s->active) return LBX_ERR_STATE;
  if (!h_n || cap < 0 || (cap > 0 && (!h_cell || !h_dir || !h_sph))) return LBX_ERR_ARG;
  // after a step pos[pcur] holds the new positions and pos[1 - pcur] those
  // of the step; lbx_set_particles wrote both slots
  const double* pos = s->pos[1 - s->pcur];
  const int8_t* fl = c.flags[s->flags_last];
  PDev P = pdev(c);
  Geom g = geom(c);
  unsigned long long* d_count = nullptr;
  if (cudaMalloc(&d_count, sizeof(*d_count)) != cudaSuccess) return LBX_ERR_ALLOC;
  cudaMemsetAsync(d_count, 0, sizeof(*d_count), c.stream);
  k_links<<<s->np, 256, 0, c.stream>>>(P, pos, g, fl, d_count, 0, nullptr, nullptr, nullptr);
  unsigned long long total = 0;
  cudaMemcpyAsync(&total, d_count, sizeof(total), cudaMemcpyDeviceToHost, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess) {
    cudaFree(d_count);
    return LBX_ERR_CUDA;
  }
  *h_n = int64_t(total);
  int rc = 0;
  if (cap > 0 && total > 0) {
    const size_t nt = size_t(total);
    int *d_cell = nullptr, *d_sph = nullptr;
    int8_t* d_dir = nullptr;
    if (cudaMalloc(&d_cell, nt * 4) != cudaSuccess || cudaMalloc(&d_sph, nt * 4) != cudaSuccess ||
        cudaMalloc(&d_dir, nt) != cudaSuccess) {
      rc = LBX_ERR_ALLOC;
    } else {
      cudaMemsetAsync(d_count, 0, sizeof(*d_count), c.stream);
      k_links<<<s->np, 256, 0, c.stream>>>(P, pos, g, fl, d_count, (long long)nt, d_cell, d_dir, d_sph);
      std::vector<int> cell(nt), sph(nt);
      std::vector<int8_t> dir(nt);
      cudaMemcpyAsync(cell.data(), d_cell, nt * 4, cudaMemcpyDeviceToHost, c.stream);
      cudaMemcpyAsync(sph.data(), d_sph, nt * 4, cudaMemcpyDeviceToHost, c.stream);
      cudaMemcpyAsync(dir.data(), d_dir, nt, cudaMemcpyDeviceToHost, c.stream);
      if (cudaStreamSynchronize(c.stream) != cudaSuccess) {
        rc = LBX_ERR_CUDA;
      } else {
        std::vector<size_t> ord(nt);
        for (size_t i = 0; i < nt; ++i) ord[i] = i;
        std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
          if (sph[x] != sph[y]) return sph[x] < sph[y];
          if (cell[x] != cell[y]) return cell[x] < cell[y];
          return dir[x] < dir[y];
        });
        const size_t m = std::min(nt, size_t(cap));
        for (size_t i = 0; i < m; ++i) {
          h_cell[i] = cell[ord[i]];
          h_dir[i] = dir[ord[i]];
          h_sph[i] = sph[ord[i]];
        }
      }
    }
    if (d_cell) cudaFree(d_cell);
    if (d_sph) cudaFree(d_sph);
    if (d_dir) cudaFree(d_dir);
  }
  cudaFree(d_count);
  if (!rc) rc = launch_status();
  return rc;
}

int particles_flags_slot(const Ctx& c) { return c.part ? c.part->flags_last : c.fcur; }
int particles_active(const Ctx& c) { return c.part && c.part->active; }

}  // namespace lbx
