// lbx_common.cuh — lattice tables, storage traits and the device error word
// shared by the sm_100a kernels of the LBcuda hot path.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/lbx.h"

namespace lbx {

constexpr int Q = 19;   // D3Q19, reference default (defines.h:8 `noD3Q27`)
constexpr int Q27 = 27; // gradient / belt neighbourhood (dimensions_m.CUF:275-281)

// Lattice velocities in the reference order (dimensions_m.CUF:211-218, and
// :130-135 for the D3Q27 build, whose first 19 directions are D3Q19's).  They
// are compile-time constants here so that every unrolled loop folds them.
__host__ __device__ constexpr int ex(int l) {
  constexpr int t[Q27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
  return t[l];
}
__host__ __device__ constexpr int ey(int l) {
  constexpr int t[Q27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1};
  return t[l];
}
__host__ __device__ constexpr int ez(int l) {
  constexpr int t[Q27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};
  return t[l];
}
__host__ __device__ constexpr int ex27(int l) {
  constexpr int t[Q27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
  return t[l];
}
__host__ __device__ constexpr int ey27(int l) {
  constexpr int t[Q27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, -1, 1};
  return t[l];
}
__host__ __device__ constexpr int ez27(int l) {
  constexpr int t[Q27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};
  return t[l];
}
// weight class of a D3Q19 direction: 0 rest, 1 axis, 2 face diagonal
__host__ __device__ constexpr int wclass(int l) { return l == 0 ? 0 : (l <= 6 ? 1 : 2); }
// weight class of a D3Q27 direction: 0..3 = number of non-zero components
__host__ __device__ constexpr int wclass27(int l) { return l == 0 ? 0 : (l <= 6 ? 1 : (l <= 18 ? 2 : 3)); }
// |e_l| class for the recolouring cosine: 0, 1, sqrt(2)
__host__ __device__ constexpr int opp(int l) { return l == 0 ? 0 : ((l & 1) ? l + 1 : l - 1); }

// Runtime tables, computed on the host in the arithmetic of the precision they
// are used in (the reference evaluates its `parameter` expressions in FP32,
// dimensions_m.CUF:201-300) and passed to kernels by value.
template <typename C>
struct LatticeT {
  C w[4];        // p_l per weight class (class 3: D3Q27 corners)
  C b[4];        // b_l classes (D3Q19: Leclaire, b_xi = 0.5; D3Q27: Saito)
  C a27[4];      // ad3q27 classes (0, p1/cssq, p2/cssq, p3/cssq)
  C p27[4];      // pd3q27 classes (D3Q27 weights, dimensions_m.CUF:283-290)
  C rec[4];      // rec_fact classes: 0, 1, sqrt(2), sqrt(3)
  C cssq;        // 1/3
  C inv_cssq;    // 1/cssq
  C half_inv_cssq;  // HALF/cssq
};

// q = 19 (default, dimensions_m.CUF:201-261) or 27 (the D3Q27 build, :117-198)
template <typename C>
inline LatticeT<C> make_lattice(int q = Q) {
  LatticeT<C> L;
  const C ONE = 1, TWO = 2, THREE = 3, SIX = 6, TWELVE = 12, TWENTYFOUR = 24;
  L.cssq = C(1.0) / C(3.0);
  L.w[0] = C(1.0) / C(3.0);
  L.w[1] = C(1.0) / C(18.0);
  L.w[2] = C(1.0) / C(36.0);
  L.w[3] = C(0);
  const C b_xi = C(0.5);
  L.b[0] = -(TWO + TWO * b_xi) / (THREE * b_xi + TWELVE);
  L.b[1] = (b_xi) / (SIX * b_xi + TWENTYFOUR);
  L.b[2] = ONE / (SIX * b_xi + TWENTYFOUR);
  L.b[3] = C(0);
  const C q1 = (TWO / THREE) * (TWO / THREE) * (ONE / SIX);
  const C q2 = (ONE / SIX) * (ONE / SIX) * (TWO / THREE);
  const C q3 = (ONE / SIX) * (ONE / SIX) * (ONE / SIX);
  L.p27[0] = (TWO / THREE) * (TWO / THREE) * (TWO / THREE);
  L.p27[1] = q1;
  L.p27[2] = q2;
  L.p27[3] = q3;
  L.a27[0] = 0;
  L.a27[1] = q1 / L.cssq;
  L.a27[2] = q2 / L.cssq;
  L.a27[3] = q3 / L.cssq;
  L.rec[0] = 0;
  L.rec[1] = 1;
  L.rec[2] = sqrt(C(2));
  L.rec[3] = sqrt(C(3));
  if (q == Q27) {  // D3Q27 weights and Saito's b_l (dimensions_m.CUF:124-143)
    for (int k = 0; k < 4; ++k) L.w[k] = L.p27[k];
    L.b[0] = -(C(10) / C(27));
    L.b[1] = TWO / C(27);
    L.b[2] = ONE / C(54);
    L.b[3] = ONE / C(216.0);
  }
  L.inv_cssq = ONE / L.cssq;
  L.half_inv_cssq = C(0.5) / L.cssq;
  return L;
}

// ---- storage traits --------------------------------------------------------
// FP16/BF16 hold f_l - w_l * rho0 (the shifted populations); arithmetic is FP32.
template <typename S> struct Store;
template <> struct Store<float> {
  using C = float;
  static __device__ __forceinline__ float ld(const float* p, float) { return __ldg(p); }
  static __device__ __forceinline__ void st(float* p, float v, float) { *p = v; }
  static __device__ __forceinline__ float enc(float v, float) { return v; }
  static __device__ __forceinline__ float dec(float h, float) { return h; }
  static constexpr bool shifted = false;
};
template <> struct Store<double> {
  using C = double;
  static __device__ __forceinline__ double ld(const double* p, double) { return __ldg(p); }
  static __device__ __forceinline__ void st(double* p, double v, double) { *p = v; }
  static __device__ __forceinline__ double enc(double v, double) { return v; }
  static __device__ __forceinline__ double dec(double h, double) { return h; }
  static constexpr bool shifted = false;
};
template <> struct Store<__half> {
  using C = float;
  static __device__ __forceinline__ float ld(const __half* p, float s) { return __half2float(__ldg(p)) + s; }
  static __device__ __forceinline__ void st(__half* p, float v, float s) { *p = __float2half_rn(v - s); }
  static __device__ __forceinline__ __half enc(float v, float s) { return __float2half_rn(v - s); }
  static __device__ __forceinline__ float dec(__half h, float s) { return __half2float(h) + s; }
  static constexpr bool shifted = true;
};
template <> struct Store<__nv_bfloat16> {
  using C = float;
  static __device__ __forceinline__ float ld(const __nv_bfloat16* p, float s) { return __bfloat162float(__ldg(p)) + s; }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float v, float s) { *p = __float2bfloat16_rn(v - s); }
  static __device__ __forceinline__ __nv_bfloat16 enc(float v, float s) { return __float2bfloat16_rn(v - s); }
  static __device__ __forceinline__ float dec(__nv_bfloat16 h, float s) { return __bfloat162float(h) + s; }
  static constexpr bool shifted = true;
};

// Shift of direction l of component c: w_l * rho0_c (zero for unshifted types).
template <typename C>
struct Shift {
  C s[2][4];  // [component][weight class]
  int sd = 0;  // sum / difference pairs: component 0 holds R + B, 1 holds R - B (s: their shifts)
  // sum / predicted-split pairs: component 1 holds E = (R - B) - split[y] (R + B) for the cell y
  // that pulls the pair; split is the phase field of each cell, or nullptr for the other formats
  const float* split = nullptr;
  __device__ __forceinline__ C at(int c, int l) const { return s[c][wclass27(l)]; }
};

// ---- geometry ---------------------------------------------------------------
// Population layout: element (l * n + cell) * nc + comp, i.e. the
// components of one direction and cell are adjacent (a half2 / float2 / double2
// for the two colour-gradient components), direction planes of n cells, x
// fastest inside a plane.
struct Geom {
  int nx, ny, nz;
  int64_t n;  // nx*ny*nz cells per direction plane
  int nc;     // components (1 BGK, 2 colour gradient)
};

__host__ __device__ __forceinline__ size_t pidx(const Geom& g, int comp, int l, int64_t cell) {
  return (size_t(l) * size_t(g.n) + size_t(cell)) * size_t(g.nc) + size_t(comp);
}

// ---- device error word -------------------------------------------------------
// One 64-bit word: [63:56] code, [55:32] step (mod 2^24), [31:0] cell/particle.
// The first error wins (atomicCAS from zero), like the reference's stop_d.
__device__ __forceinline__ void raise_error(unsigned long long* err, int code, int64_t step, int64_t where) {
  unsigned long long v = (static_cast<unsigned long long>(code & 0xff) << 56) |
                         ((static_cast<unsigned long long>(step) & 0xffffffull) << 32) |
                         (static_cast<unsigned long long>(where) & 0xffffffffull);
  atomicCAS(err, 0ull, v);
}

}  // namespace lbx
