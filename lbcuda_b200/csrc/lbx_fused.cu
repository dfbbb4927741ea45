// lbx_fused.cu — single-pass colour-gradient step (time_step_CG + streaming,
// kernels_fluid_CG.CUF:531-1141) for sm_100a, written for instruction
// economy: the two components of a direction are one 4- or 8-byte word in
// memory, the collision relaxes their sum (the recolouring needs nothing
// else when the colour gradient is non-zero), a direction and its opposite
// form one packed FP32 pair for the sm_100 add / mul / fma .f32x2
// instructions (e_opp = -e_l, so every odd power of e.u / e.psi changes sign
// and every even power is shared), 16-bit values enter the FP32 sums by
// mixed-precision adds, and all per-class products (omega rho w_l, the
// perturbation and recolouring coefficients) are formed once per cell.
//
// Schedule: a CTA of TX x TY threads owns the column [x0, x0+TX) x [y0, y0+TY)
// and marches it along z over one segment (32 planes by default).  In
// iteration z it
//   1. starts the pulls of plane z+2 for its own cells and the one-cell ring
//      around the column: 16-bit storage copies them into a three-plane
//      shared-memory stage by cp.async (FP32 / FP64 pull synchronously in
//      step 2 instead);
//   2. sums the pulls of plane z+1 (landed one iteration ago) into densities
//      and writes their phase field into a rolling window (two planes with
//      staged pulls, four otherwise), then arrives at the plane's split
//      barrier (an mbarrier);
//   3. reads the pairs of plane z from the stage and relaxes their component
//      sums (BGK half), waits at the barrier, takes the colour gradient
//      (staged: the in-plane sums of plane z+1 from the window, those of z-1
//      and z kept in registers; otherwise the 26-point sum, its planes z-1
//      and z before the wait), perturbs and recolours, and stores the 38
//      post-collision values of each cell with coalesced 4- or 8-byte writes.
// The phase field never goes through global memory; the extra cost is the
// ring and the two boundary planes of each segment.  The particle variant
// (PART) also copies each cell's flag words and side phase field with its
// pulls and collides only fluid cells.
#include "lbx_device.cuh"

#include <algorithm>
#include <type_traits>
#include <utility>
#include <vector>

namespace lbx {

// f(std::integral_constant<int, l>) for the even / odd directions l of D3Q19,
// each with its direction as a compile-time constant
template <typename F, int... I>
__device__ __forceinline__ void unroll_dirs(F& f, int first, std::integer_sequence<int, I...>) {
  (void)first;
  (f(std::integral_constant<int, 2 * I>{}), ...);
}
template <typename F, int... I>
__device__ __forceinline__ void unroll_dirs_odd(F& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, 2 * I + 1>{}), ...);
}
template <typename F>
__device__ __forceinline__ void unroll_even(F& f) { unroll_dirs(f, 0, std::make_integer_sequence<int, 10>{}); }
template <typename F>
__device__ __forceinline__ void unroll_odd(F& f) { unroll_dirs_odd(f, std::make_integer_sequence<int, 9>{}); }

template <typename C>
struct LeanConst {
  C w[3], b[3], a27[4];
  C sqrt2;
  C w2_sqrt2;        // w_2 / sqrt 2 (recolouring weight of the face diagonals)
  C omega;           // uniform relaxation (tauR == tauB), else negative
  C inv_viscR, inv_viscB, inv_cssq;
  C sigma, beta;
  C rho0[2];         // shift densities of the stored populations (0 when unshifted)
  C s[2][3];         // shift of each weight class, w_cls * rho0
  // sum / difference pairs (LBX_STORE_F16_SD, _BF16_SD): the stored pair is
  // (R + B, R - B) less these shifts
  C rho0sd[2];       // rho0R + rho0B, rho0R - rho0B
  C ssd[2][3];       // w_cls * rho0sd
};

template <typename C>
LeanConst<C> make_lean(const Ctx& c) {
  LeanConst<C> K;
  LatticeT<C> L = make_lattice<C>();
  for (int i = 0; i < 3; ++i) { K.w[i] = L.w[i]; K.b[i] = L.b[i]; }
  for (int i = 0; i < 4; ++i) K.a27[i] = L.a27[i];
  K.sqrt2 = L.rec[2];
  K.w2_sqrt2 = K.w[2] / K.sqrt2;
  const C HALF = C(0.5);
  C viscR = L.cssq * (C(c.p.tauR) - HALF), viscB = L.cssq * (C(c.p.tauB) - HALF);
  K.inv_viscR = C(1) / viscR;
  K.inv_viscB = C(1) / viscB;
  K.inv_cssq = L.inv_cssq;
  K.omega = (c.p.tauR == c.p.tauB) ? C(1) / (viscR / L.cssq + HALF) : C(-1);
  K.sigma = C(c.p.sigma);
  K.beta = C(c.p.beta);
  bool shifted = c.storage != LBX_STORE_F32 && c.storage != LBX_STORE_F64;
  K.rho0[0] = shifted ? C(c.p.rho0R) : C(0);
  K.rho0[1] = shifted ? C(c.p.rho0B) : C(0);
  K.rho0sd[0] = K.rho0[0] + K.rho0[1];
  K.rho0sd[1] = c.sdp ? C(0) : K.rho0[0] - K.rho0[1];  // the predicted split's deviation is stored unshifted
  for (int comp = 0; comp < 2; ++comp)
    for (int k = 0; k < 3; ++k) {
      K.s[comp][k] = K.w[k] * K.rho0[comp];
      K.ssd[comp][k] = K.w[k] * K.rho0sd[comp];
    }
  return K;
}

// raw stored value -> arithmetic type (no shift)
template <typename S> __device__ __forceinline__ float raw(S v);
template <> __device__ __forceinline__ float raw<float>(float v) { return v; }
template <> __device__ __forceinline__ float raw<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float raw<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ double raw_d(double v) { return v; }

template <typename S, typename C>
__device__ __forceinline__ C load_raw(const S* p) {
  if constexpr (std::is_same<S, double>::value) return __ldg(p);
  else return raw<S>(__ldg(p));
}
template <typename S, typename C>
__device__ __forceinline__ void store_raw(S* p, C v) {
  if constexpr (std::is_same<S, double>::value || std::is_same<S, float>::value) *p = v;
  else if constexpr (std::is_same<S, __half>::value) *p = __float2half_rn(v);
  else *p = __float2bfloat16_rn(v);
}

// 32-bit source offsets of the 19 pulls of a cell
struct PullIdx {
  int src[Q];
};

__device__ __forceinline__ void pull_idx(const Geom& g, int x, int y, int z, PullIdx& P) {
  int xm = (x == 0) ? g.nx - 1 : x - 1, xp = (x == g.nx - 1) ? 0 : x + 1;
  int ym = (y == 0) ? g.ny - 1 : y - 1, yp = (y == g.ny - 1) ? 0 : y + 1;
  int zm = (z == 0) ? g.nz - 1 : z - 1, zp = (z == g.nz - 1) ? 0 : z + 1;
  const int X[3] = {xm, x, xp};
  const int Y[3] = {ym * g.nx, y * g.nx, yp * g.nx};
  const int plane = g.nx * g.ny;
  const int Z[3] = {zm * plane, z * plane, zp * plane};
#pragma unroll
  for (int l = 0; l < Q; ++l) P.src[l] = X[1 - ex(l)] + Y[1 - ey(l)] + Z[1 - ez(l)];
}

// source offset of the pull of direction l alone (the same wrap as
// pull_idx; a caller that needs all 19 at once lets the compiler share the
// neighbour coordinates, and nothing stays live between two uses)
__device__ __forceinline__ int pull_one(const Geom& g, int x, int y, int z, int l) {
  const int sx = ex(l) == 0 ? x : (ex(l) > 0 ? (x == 0 ? g.nx - 1 : x - 1) : (x == g.nx - 1 ? 0 : x + 1));
  const int sy = ey(l) == 0 ? y : (ey(l) > 0 ? (y == 0 ? g.ny - 1 : y - 1) : (y == g.ny - 1 ? 0 : y + 1));
  const int sz = ez(l) == 0 ? z : (ez(l) > 0 ? (z == 0 ? g.nz - 1 : z - 1) : (z == g.nz - 1 ? 0 : z + 1));
  return sx + g.nx * (sy + g.ny * sz);
}

// ---- component pairs ---------------------------------------------------------
// The two components of one direction and cell are adjacent in memory, so one
// load / store moves both; in registers they form one float2 on which the
// sm_100 packed FP32 instructions (add / mul / fma .f32x2) act.
template <typename C> struct PairT;
template <> struct PairT<float> { using T = float2; };
template <> struct PairT<double> { using T = double2; };
template <typename C> using P2 = typename PairT<C>::T;

__device__ __forceinline__ float2 pp(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pp(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 p_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 p_mul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 p_fma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}

// a + c for a 16-bit a and an FP32 c, rounded once (sm_100 mixed-precision
// add: the conversion of a is exact, so this equals float(a) + c)
__device__ __forceinline__ float add_mixed(__half a, float c) {
  float d;
  asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(__half_as_ushort(a)), "f"(c));
  return d;
}
__device__ __forceinline__ float add_mixed(__nv_bfloat16 a, float c) {
  float d;
  asm("add.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(__bfloat16_as_ushort(a)), "f"(c));
  return d;
}

// storage pair <-> arithmetic pair (R: the stored pair as one word)
template <typename S> struct SPair;
template <> struct SPair<float> {
  using R = float2;
  static __device__ __forceinline__ R ldr(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
  static __device__ __forceinline__ float2 cvt(R r) { return r; }
  static __device__ __forceinline__ float sum(R r) { return r.x + r.y; }
  static __device__ __forceinline__ float first(R r) { return r.x; }
  static __device__ __forceinline__ float2 ld(const float* p) { return cvt(ldr(p)); }
  static __device__ __forceinline__ void st(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
};
template <> struct SPair<double> {
  using R = double2;
  static __device__ __forceinline__ R ldr(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
  static __device__ __forceinline__ double2 cvt(R r) { return r; }
  static __device__ __forceinline__ double sum(R r) { return r.x + r.y; }
  static __device__ __forceinline__ double first(R r) { return r.x; }
  static __device__ __forceinline__ double2 ld(const double* p) { return cvt(ldr(p)); }
  static __device__ __forceinline__ void st(double* p, double2 v) { *reinterpret_cast<double2*>(p) = v; }
};
template <> struct SPair<__half> {
  using R = __half2;
  static __device__ __forceinline__ R ldr(const __half* p) { return __ldg(reinterpret_cast<const __half2*>(p)); }
  static __device__ __forceinline__ float2 cvt(R r) { return __half22float2(r); }
  static __device__ __forceinline__ float sum(R r) { return add_mixed(r.y, __low2float(r)); }
  static __device__ __forceinline__ float first(R r) { return __low2float(r); }
  static __device__ __forceinline__ float2 ld(const __half* p) { return cvt(ldr(p)); }
  static __device__ __forceinline__ void st(__half* p, float2 v) {
    *reinterpret_cast<__half2*>(p) = __float22half2_rn(v);
  }
};
template <> struct SPair<__nv_bfloat16> {
  using R = __nv_bfloat162;
  static __device__ __forceinline__ R ldr(const __nv_bfloat16* p) {
    return __ldg(reinterpret_cast<const __nv_bfloat162*>(p));
  }
  static __device__ __forceinline__ float2 cvt(R r) { return __bfloat1622float2(r); }
  static __device__ __forceinline__ float sum(R r) { return add_mixed(r.y, __low2float(r)); }
  static __device__ __forceinline__ float first(R r) { return __low2float(r); }
  static __device__ __forceinline__ float2 ld(const __nv_bfloat16* p) { return cvt(ldr(p)); }
  static __device__ __forceinline__ void st(__nv_bfloat16* p, float2 v) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
  }
};

// Which pulls land in shared memory by cp.async ("staged"): the 4-byte pairs
// of 16-bit storage.  FP32 and FP64 pull synchronously and re-read the pairs
// from L2 for the collision: a two-deep FP32 stage (109 KB per CTA, issued
// once the collision has read a plane's pairs) measured 0.235 ms at 128^3
// against 0.156 ms without it.  Own-cell pairs are 3 planes deep: plane z+2
// is copied at the top of iteration z.  Copying one plane further ahead (4
// planes, 100 KB per CTA) measured 0.165 ms against 0.107 at FP16 128^3: the
// larger stage leaves the L1 too small for the pulls.
template <typename S, bool PART>
constexpr bool kStaged = sizeof(typename SPair<S>::R) == 4;
template <typename S, bool PART>
constexpr int kDepth = 3;

// element offset of direction l (both components) of a cell: 2 (l n + cell)
__device__ __forceinline__ size_t poff(int64_t n, int l, int cell) { return (size_t(l) * size_t(n) + size_t(cell)) * 2; }

// Direction plane l of a population buffer: its pair of cell c is at
// plane(l)[2 c].  The plane base is the same for every thread, so each access
// costs one 32-bit index scaled onto a uniform base.
template <typename S>
struct Planes {
  S* p;
  int64_t n2;  // 2 n elements per direction plane
  __device__ __forceinline__ S* operator()(int l) const { return p + size_t(l) * size_t(n2); }
  // pair i of direction plane l; the unsigned index keeps the per-thread part
  // one 32 x 32 -> 64-bit multiply-add onto the plane base (a signed int
  // index measured 84 more integer instructions per cell)
  __device__ __forceinline__ S* at(int l, int i) const { return (*this)(l) + 2 * size_t(unsigned(i)); }
};

// ---- asynchronous copies global -> shared (cp.async, 4-byte granules) --------
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <typename C>
__device__ __forceinline__ void cp_async_c(C* smem, const C* gmem) {
  if constexpr (sizeof(C) == 4) cp_async4(smem, gmem);
  else cp_async8(smem, gmem);
}
// 16-byte granule, L2 -> shared memory without an L1 allocation
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- split barrier of a plane (mbarrier in shared memory) -----------------
// Every thread arrives once the phase field of plane z+1 is in the window and
// waits only before its collision reads that plane, so the BGK half of the
// collision runs while slower threads finish their copies.
__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(m));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* m) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(m));
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(a) : "memory");
}
// arrive on the barrier once every cp.async this thread has issued so far has
// landed (the barrier's expected count includes this arrival)
__device__ __forceinline__ void mbar_arrive_cp_async(unsigned long long* m) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(m));
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(a) : "memory");
}
// wait for the completion of the phase of the given parity; false if the
// bounded number of polls ran out (each poll may itself suspend a while)
__device__ __forceinline__ bool mbar_wait(unsigned long long* m, unsigned parity) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(m));
  for (int i = 0; i < (1 << 22); ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// issue the 19 pulls of a cell as asynchronous copies into st[l * stride]
template <typename S>
__device__ __forceinline__ void pull_async(const S* __restrict__ A, int64_t n, const PullIdx& P,
                                           typename SPair<S>::R* st, int stride) {
  static_assert(sizeof(typename SPair<S>::R) == 4 || sizeof(typename SPair<S>::R) == 8, "4- or 8-byte pairs");
  const Planes<const S> Ap{A, 2 * n};
#pragma unroll
  for (int l = 0; l < Q; ++l) {
    if constexpr (sizeof(typename SPair<S>::R) == 4) cp_async4(st + l * stride, Ap.at(l, P.src[l]));
    else cp_async8(st + l * stride, Ap.at(l, P.src[l]));
  }
}

// densities (Sum g + rho0, before the clamp) from pairs already in shared
// memory: each 16-bit value is added to the FP32 sums by one mixed-precision
// add (same order and roundings as converting first).  SD: the pairs are
// (R + B, R - B), whose sums give rho and rhoR - rhoB.
// at(l): the staged pair of direction l
template <typename S, typename C, bool SD = false, bool SDP = false, typename F>
__device__ __forceinline__ void stage_rho(F&& at, const LeanConst<C>& K, C& rR, C& rB, C split = C(0)) {
  P2<C> s = SPair<S>::cvt(at(0));
#pragma unroll
  for (int l = 1; l < Q; ++l) {
    const typename SPair<S>::R r = at(l);
    s.x = add_mixed(r.x, s.x);
    s.y = add_mixed(r.y, s.y);
  }
  if constexpr (SD) {
    // predicted split: Sum (R - B) = Sum E + split Sum (R + B)
    const C rho = s.x + K.rho0sd[0], dif = SDP ? fma(split, rho, s.y) : s.y + K.rho0sd[1];
    rR = C(0.5) * (rho + dif);
    rB = C(0.5) * (rho - dif);
  } else {
    rR = s.x + K.rho0[0];
    rB = s.y + K.rho0[1];
  }
}

// densities (Sum g + rho0, init_rho*_CG, before the clamp) of the pulled
// cell; with a stage, the pulled pairs are also kept there (direction l at
// st[l * stride]) for the collision of the same cell one plane later
template <typename S, typename C>
__device__ __forceinline__ void pull_rho(const S* __restrict__ A, int64_t n, const PullIdx& P, const LeanConst<C>& K,
                                         C& rR, C& rB, typename SPair<S>::R* st = nullptr, int stride = 0) {
  const Planes<const S> Ap{A, 2 * n};
  typename SPair<S>::R r = SPair<S>::ldr(Ap(0) + 2 * P.src[0]);
  if (st) st[0] = r;
  P2<C> s = SPair<S>::cvt(r);
#pragma unroll
  for (int l = 1; l < Q; ++l) {
    r = SPair<S>::ldr(Ap.at(l, P.src[l]));
    if (st) st[l * stride] = r;
    s = p_add(s, SPair<S>::cvt(r));
  }
  rR = s.x + K.rho0[0];
  rB = s.y + K.rho0[1];
}

template <typename C>
__device__ __forceinline__ C clamp0(C v) { return v < C(0) ? C(0) : v; }

// a * b + c with one rounding.  This file is compiled without automatic
// contraction (-fmad=false): every fused operation is written out, so each
// kernel that inlines the collision rounds identically.
template <typename C>
__device__ __forceinline__ C fm(C a, C b, C c) { return fma(a, b, c); }

// reciprocal (FP32: the hardware approximation rcp.approx.ftz, within 1 ulp;
// the correctly rounded __frcp_rn measured 3.5 % slower at FP16 128^3) and
// reciprocal square root (FP32: rsqrtf)
template <typename C>
__device__ __forceinline__ C rcp_c(C x) {
  if constexpr (sizeof(C) == 4) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else return C(1) / x;
}
template <typename C>
__device__ __forceinline__ C rsqrt_c(C x) {
  if constexpr (sizeof(C) == 4) return rsqrtf(x);
  else return C(1) / sqrt(x);
}
// phase field (rR - rB) / (rR + rB)
template <typename C>
__device__ __forceinline__ C phase_of(C rR, C rB) { return (rR - rB) * rcp_c(rR + rB); }

// One colour-gradient collision (time_step_CG, kernels_fluid_CG.CUF:689-846)
// in two halves around the plane barrier, written on component SUMS.  When
// the colour gradient is non-zero the recolouring needs, per direction, only
// fd_l = f'_R,l + f'_B,l + perturbation (the BGK-relaxed sum) and the cell's
// densities: the relaxed components themselves are never used.  So the BGK
// half relaxes S_l = g_R,l + g_B,l (stored form; the shifts fold into one
// constant per weight class),
//   h_l = f'_R,l + f'_B,l = (1 - omega) S_l + omega rho w_l A_l(u) + (1 - omega) s_l,
// and the recolouring half forms both outputs from h_l.  A direction pair
// (l, opposite) is one packed FP32 pair: e_opp = -e_l, so (e.u, -e.u) and
// (e.psi, -e.psi) give both directions' A, perturbation and recolouring term
// from the same packed instructions.  A cell without a colour gradient
// (|psi|^2 <= 1e-20) keeps the per-component BGK result (bgk_components).
template <typename C>
struct Relaxed {
  C h0;         // rest direction
  P2<C> h[9];   // pair p: (h_{2p-1}, h_{2p})
  C u, v, w, c0, omega, inv;
};

// packed pair (e.a, -e.a) of direction 2p-1 from the pairs (a_i, -a_i) and (-a_i, a_i)
template <typename C>
__device__ __forceinline__ P2<C> edot_pair(int l, const P2<C> pos[3], const P2<C> neg[3]) {
  const int e[3] = {ex(l), ey(l), ez(l)};
  P2<C> r = pp(C(0), C(0));
  bool any = false;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (!e[i]) continue;
    const P2<C> t = e[i] > 0 ? pos[i] : neg[i];
    r = any ? p_add(r, t) : t;
    any = true;
  }
  return r;
}

// BGK half: S[l] = g_R,l + g_B,l of the pulled (stored-form) pairs; rR/rB: clamped densities
template <typename C>
__device__ __forceinline__ Relaxed<C> relax_sums(const LeanConst<C>& K, const C S[Q], C rR, C rB, bool shifted) {
  const C ONE = C(1), HALF = C(0.5);
  const C rs = rR + rB;
  Relaxed<C> X;
  C omega;
  if (K.omega >= C(0)) {
    omega = K.omega;
  } else {
    const C ph = (rR - rB) / rs;
    const C visc = ONE / (HALF * (ONE + ph) * K.inv_viscR + HALF * (ONE - ph) * K.inv_viscB);
    omega = ONE / fm(visc, K.inv_cssq, HALF);
  }
  const C omm = ONE - omega;
  const C inv = rcp_c(rs);
  // momentum from the opposite-pair differences (shifts cancel)
  C mu = C(0), mv = C(0), mw = C(0);
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int l = 2 * p - 1;
    const C d = S[l] - S[l + 1];
    if (ex(l)) mu = ex(l) > 0 ? mu + d : mu - d;
    if (ey(l)) mv = ey(l) > 0 ? mv + d : mv - d;
    if (ez(l)) mw = ez(l) > 0 ? mw + d : mw - d;
  }
  const C u = inv * mu, v = inv * mv, w = inv * mw;
  const C c0 = fm(C(-1.5), fm(u, u, fm(v, v, w * w)), ONE);
  // per weight class: omega rho w and the folded shift (1 - omega) (s_R + s_B)
  C kc[3], hs[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    kc[k] = omega * rs * K.w[k];
    hs[k] = shifted ? omm * (K.s[0][k] + K.s[1][k]) : C(0);
  }
  X.h0 = shifted ? fm(omm, S[0], fm(kc[0], c0, hs[0])) : fm(omm, S[0], kc[0] * c0);
  const P2<C> pos[3] = {pp(u, -u), pp(v, -v), pp(w, -w)};
  const P2<C> neg[3] = {pp(-u, u), pp(-v, v), pp(-w, w)};
  const P2<C> OMM = pp(omm, omm), C0 = pp(c0, c0), F45 = pp(C(4.5), C(4.5)), THREE = pp(C(3), C(3));
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int l = 2 * p - 1, k = wclass(l);
    const P2<C> eu = edot_pair<C>(l, pos, neg);            // (e.u, -e.u)
    const P2<C> P = p_fma(p_mul(F45, eu), eu, C0);        // 1 + 4.5 (e.u)^2 - 1.5 u^2
    const P2<C> A = p_fma(THREE, eu, P);                  // + 3 e.u, - 3 e.u
    const P2<C> Sv = pp(S[l], S[l + 1]);
    const P2<C> KC = pp(kc[k], kc[k]);
    X.h[p - 1] = shifted ? p_fma(OMM, Sv, p_fma(KC, A, pp(hs[k], hs[k]))) : p_fma(OMM, Sv, p_mul(KC, A));
  }
  X.u = u;
  X.v = v;
  X.w = w;
  X.c0 = c0;
  X.omega = omega;
  X.inv = inv;
  return X;
}

// Recolouring half (perturbation + recolouring): the post-collision pairs
// (stored form) into out[]; false, with out[] untouched, when the colour
// gradient is below the reference's limit.  SD: the pairs (R + B, R - B)
// less their shifts; R + B is the perturbed total itself (kR + kB = 1 up to
// rounding, the recolouring terms cancel) and R - B = (kR - kB) f + 2 T.
template <typename C, bool SD = false, bool SDP = false, int RXW = 0>
__device__ __forceinline__ bool recolour_sums(const LeanConst<C>& K, const Relaxed<C>& X, C rR, C rB, C px, C py,
                                              C pz, bool shifted, P2<C> out[Q], const C* const* win = nullptr,
                                              int own = 0) {
  const C psq = fm(px, px, fm(py, py, pz * pz));
  if (!(psq > C(1.e-20))) return false;
  const C ipn = rsqrt_c(psq);
  const C pn = psq * ipn;
  const C acoeff = C(9) / C(4) * X.omega * K.sigma;
  const C coef = K.beta * rR * rB * X.inv * ipn;  // beta rR rB / (rs |psi|)
  const C kR = rR * X.inv, kB = rB * X.inv;
  C K1[3], K0[3], K3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    K1[k] = acoeff * K.w[k] * ipn;  // acoeff |psi| w / |psi|^2
    K0[k] = acoeff * pn * K.b[k];
  }
  K3[0] = C(0);
  K3[1] = coef * K.w[1];
  K3[2] = coef * K.w2_sqrt2;
  const P2<C> KK = pp(kR, kB);
  if constexpr (SD) {
    const C kD = kR - kB;
    const C fd = X.h0 - K0[0];
    // predicted split: the difference is stored as its deviation from the
    // split of the receiving cell x + e_l (its phase field, win[1 + e_lz]
    // at own + e_ly RX + e_lx), i.e. with the coefficient kD - phi_dest
    auto dest = [&](int l) -> C { return win[1 + ez(l)][own + ey(l) * RXW + ex(l)]; };
    out[0] = pp(fd - K.ssd[0][0], fm(SDP ? kD - dest(0) : kD, fd, -K.ssd[1][0]));
    const P2<C> pos[3] = {pp(px, -px), pp(py, -py), pp(pz, -pz)};
    const P2<C> neg[3] = {pp(-px, px), pp(-py, py), pp(-pz, pz)};
    const P2<C> KD = pp(kD, kD);
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      const int l = 2 * p - 1, k = wclass(l);
      const P2<C> ed = edot_pair<C>(l, pos, neg);                              // (e.psi, -e.psi)
      const P2<C> pert = p_fma(pp(K1[k], K1[k]), p_mul(ed, ed), pp(-K0[k], -K0[k]));
      const C t2 = C(2) * K3[k];
      const P2<C> cD = p_fma(pp(t2, t2), ed, pp(-K.ssd[1][k], -K.ssd[1][k]));  // (2T, -2T) - s_D
      const P2<C> fd = p_add(X.h[p - 1], pert);
      const P2<C> oS = p_add(fd, pp(-K.ssd[0][k], -K.ssd[0][k]));
      const P2<C> oD = p_fma(SDP ? p_add(KD, pp(-dest(l), -dest(l + 1))) : KD, fd, cD);
      out[l] = pp(oS.x, oD.x);
      out[l + 1] = pp(oS.y, oD.y);
    }
    return true;
  }
  {
    const C fd = X.h0 - K0[0];
    out[0] = shifted ? p_fma(pp(fd, fd), KK, pp(-K.s[0][0], -K.s[1][0])) : p_mul(pp(fd, fd), KK);
  }
  const P2<C> pos[3] = {pp(px, -px), pp(py, -py), pp(pz, -pz)};
  const P2<C> neg[3] = {pp(-px, px), pp(-py, py), pp(-pz, pz)};
  const P2<C> KR = pp(kR, kR), KB = pp(kB, kB), NEG = pp(C(-1), C(-1));
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int l = 2 * p - 1, k = wclass(l);
    const P2<C> ed = edot_pair<C>(l, pos, neg);                              // (e.psi, -e.psi)
    const P2<C> pert = p_fma(pp(K1[k], K1[k]), p_mul(ed, ed), pp(-K0[k], -K0[k]));
    const P2<C> T = p_mul(pp(K3[k], K3[k]), ed);                             // (T, -T)
    const P2<C> fd = p_add(X.h[p - 1], pert);
    const P2<C> cR = shifted ? p_add(T, pp(-K.s[0][k], -K.s[0][k])) : T;
    const P2<C> cB = shifted ? p_fma(T, NEG, pp(-K.s[1][k], -K.s[1][k])) : p_mul(T, NEG);
    const P2<C> oR = p_fma(KR, fd, cR);
    const P2<C> oB = p_fma(KB, fd, cB);
    out[l] = pp(oR.x, oB.x);
    out[l + 1] = pp(oR.y, oB.y);
  }
  return true;
}

// BGK result per component (no colour gradient): g' = g (1 - omega) +
// omega rho_k w A(u) - omega s_k, in place on the pulled pairs g[] (R, B of
// each direction).  PACKED: a direction and its opposite packed per
// component (used with staged 16-bit pulls; the FP32 / FP64 kernels, with
// more state live at this point, keep the per-direction form and stay
// within their registers without spilling).
template <typename C, bool PACKED, bool SD = false>
__device__ __forceinline__ void bgk_components(const LeanConst<C>& K, const Relaxed<C>& X, C rR, C rB, bool shifted,
                                               P2<C> g[Q]) {
  // SD: g holds (R + B, R - B) pairs, rR / rB are rho and rhoR - rhoB, and
  // the same BGK step (linear in the populations and the densities) applies
  // with the shifts of the sum and the difference
  const C(&sh)[2][3] = SD ? K.ssd : K.s;
  const C omega = X.omega, omm = C(1) - omega;
  if constexpr (!PACKED) {
    const P2<C> omm2 = pp(omm, omm);
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      const int k = wclass(l);
      const C eu = edot(l, X.u, X.v, X.w);
      const C a = fm(C(3), eu, fm(C(4.5) * eu, eu, X.c0));
      const P2<C> kc = pp(omega * rR * K.w[k], omega * rB * K.w[k]);
      g[l] = shifted ? p_fma(g[l], omm2, p_fma(kc, pp(a, a), pp(-omega * sh[0][k], -omega * sh[1][k])))
                     : p_fma(g[l], omm2, p_mul(kc, pp(a, a)));
    }
    return;
  }
  const P2<C> OMM = pp(omm, omm), C0 = pp(X.c0, X.c0), F45 = pp(C(4.5), C(4.5)), THREE = pp(C(3), C(3));
  const P2<C> pos[3] = {pp(X.u, -X.u), pp(X.v, -X.v), pp(X.w, -X.w)};
  const P2<C> neg[3] = {pp(-X.u, X.u), pp(-X.v, X.v), pp(-X.w, X.w)};
  {
    const P2<C> kc = pp(omega * rR * K.w[0], omega * rB * K.w[0]);
    g[0] = shifted ? p_fma(g[0], OMM, p_fma(kc, C0, pp(-omega * sh[0][0], -omega * sh[1][0])))
                   : p_fma(g[0], OMM, p_mul(kc, C0));
  }
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int l = 2 * p - 1, k = wclass(l);
    const P2<C> eu = edot_pair<C>(l, pos, neg);
    const P2<C> A = p_fma(THREE, eu, p_fma(p_mul(F45, eu), eu, C0));  // (A_l, A_opp)
    const C kR = omega * rR * K.w[k], kB = omega * rB * K.w[k];
    const P2<C> Rv = pp(g[l].x, g[l + 1].x), Bv = pp(g[l].y, g[l + 1].y);
    P2<C> oR, oB;
    if (shifted) {
      oR = p_fma(Rv, OMM, p_fma(pp(kR, kR), A, pp(-omega * sh[0][k], -omega * sh[0][k])));
      oB = p_fma(Bv, OMM, p_fma(pp(kB, kB), A, pp(-omega * sh[1][k], -omega * sh[1][k])));
    } else {
      oR = p_fma(Rv, OMM, p_mul(pp(kR, kR), A));
      oB = p_fma(Bv, OMM, p_mul(pp(kB, kB), A));
    }
    g[l] = pp(oR.x, oB.x);
    g[l + 1] = pp(oR.y, oB.y);
  }
}

// In-plane parts of the D3Q27 colour gradient (HIGHGRAD, time_step_CG
// kernels_fluid_CG.CUF:720-741).  Its weights factor as
// a(e) = w27(e) / cs^2 = 3 W(ex) W(ey) W(ez) with W(0) = 2/3, W(+-1) = 1/6, so
//   psi_x = 1/2 Sum_dz W(dz) Gx(z+dz),  psi_y likewise with Gy,
//   psi_z = 1/2 (M(z+1) - M(z-1)),
// where, on one plane, Gx = Sum_dy W(dy) (phi(x+1) - phi(x-1)), Gy the same
// across y, and M = Sum_dx,dy W(dx) W(dy) phi.  Each cell forms Gx, Gy, M of
// a plane once (9 reads of the window) and keeps the last three planes'
// values in registers, instead of 26 reads and 54 products per cell.  Used
// with staged pulls; the kernels that pull FP32 / FP64 pairs synchronously
// keep the 26-point sum, whose planes z-1 and z run before the plane barrier
// and hide the latency of the collision's pulls (the separable form, all
// after the barrier, measured 0.213 ms against 0.152 at FP32 128^3).
template <typename C>
struct PlaneGrad {
  C gx, gy, m;
};

template <typename C, int RX>
__device__ __forceinline__ PlaneGrad<C> plane_grad(const C* plane, int own) {
  const C W0 = C(2) / C(3), W1 = C(1) / C(6);
  const C* r0 = plane + own;
  const C a = r0[-RX - 1], b = r0[-RX], c = r0[-RX + 1];
  const C d = r0[-1], e = r0[0], f = r0[1];
  const C g = r0[RX - 1], h = r0[RX], i = r0[RX + 1];
  PlaneGrad<C> G;
  G.gx = fm(W0, f - d, W1 * ((c - a) + (i - g)));
  G.gy = fm(W0, h - b, W1 * ((g - a) + (i - c)));
  const C lo = fm(W0, b, W1 * (a + c)), mid = fm(W0, e, W1 * (d + f)), hi = fm(W0, h, W1 * (g + i));
  G.m = fm(W0, mid, W1 * (lo + hi));
  return G;
}

template <int TX, int TY>
struct Ring {
  static constexpr int RX = TX + 2, RY = TY + 2, CELLS = RX * RY, N = 2 * RX + 2 * TY, NT = TX * TY;
};

// periodic wrap of a plane index p in [-n, 2n) (the planes a segment touches,
// z0 - 1 .. zend + 1, with n >= 3): two compares instead of a division
__device__ __forceinline__ int wrap_plane(int p, int n) { return p < 0 ? p + n : (p >= n ? p - n : p); }
__device__ __forceinline__ int wrap0(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Particle data of a step: flags of this and of the previous step, and the
// side densities of the cells that are not pulled here (new fluid cells from
// the fill kernel, surface cells from the wetting kernel).  The densities of
// the fluid cells the particle kernels read come from their own shell pass
// (k_rho_shell), so nothing is written back here.
template <typename C>
struct LeanPart {
  const int8_t* __restrict__ fold;
  const int8_t* __restrict__ fnew;
  const C* __restrict__ rhoR;
  const C* __restrict__ rhoB;
  const C* __restrict__ phi;  // phase field of the surface and new fluid cells
};

// Shared memory of one CTA: the rolling phase-field window (2 planes of the
// column and its ring with staged pulls, else 4) and, for 16-bit storage, the
// stage that the pulls land
// in by cp.async: 3 planes x Q directions x the column's cells (a plane is
// copied two iterations before its collision, summed into densities one
// iteration before, and collided from the same copy), then 2 planes x Q x
// the ring cells (summed only).
//
// The particle variant adds, per own / ring cell and plane, the side record
// copied with the pulls: the 4-byte words holding the cell's flag of this and
// of the previous step, and the phase field the wetting / fill kernels wrote
// for it (3 planes deep for own cells, 2 for ring cells).
template <typename C>
struct SideRec {
  unsigned fnew_w, fold_w;  // aligned words containing the cell's flags
  C phi;
};

// Staged pulls in boxes (BOX, 16-bit storage with nx a multiple of 4): per
// plane and direction l, the rows y0 - 1 - e_ly .. y0 + TY - e_ly and the
// columns x0 - 4 .. x0 + TX + 3 of direction plane l at z - e_lz, copied by
// 16-byte cp.async granules (a granule starts on a multiple of 4 cells, so
// the periodic wrap moves whole granules).  Own cell (tx, ty) finds its pull
// of direction l at box row ty + 1, column tx + 4 - e_lx; ring cell (rx, ry)
// at row ry, column rx + 3 - e_lx: one per-thread base and a constant offset
// per direction.  Each plane slot has a FULL barrier (every thread arrives
// once its copies have landed, cp.async.mbarrier.arrive) and an EMPTY
// barrier (every thread arrives after its last read of the plane), since a
// thread now reads what other threads copied.
template <int TX, int TY>
struct LeanBox {
  static constexpr int BW = TX + 8, ROWS = TY + 2, ELEMS = BW * ROWS;  // 4-byte pairs per direction box
  static constexpr int GR = BW / 4;                                    // granules per row
  static constexpr int POS = ROWS * GR;                                // granule positions per box
  static constexpr int NT = TX * TY;
  static constexpr int G = NT / POS;  // copy groups: group k copies directions k, k + G, ...
  static_assert(G == 2, "box copies are written for two groups (even / odd directions)");
  static constexpr int COPIERS = G * POS;
  // particle variant: the flag bytes of this and of the previous step (rows
  // y0 - 1 .. y0 + TY, bytes x0 - 16 .. x0 + TX + 15: 16-byte granules at
  // multiples of 16 cells, so nx % 16 == 0), copied by group 0, and the side
  // phase field (the pull box's rows and columns, e = 0), copied by group 1
  static constexpr int FBW = TX + 32, FGR = FBW / 16, FB = ROWS * FBW;  // bytes per row / granules / per array
  static constexpr int FPOS = 2 * ROWS * FGR;
  static_assert(FPOS <= POS, "flag granules: one per copier of group 0");
};

template <typename S, int TX, int TY, bool PART, bool SDP = false, bool BOX = false>
struct LeanSmem {
  using C = typename Store<S>::C;
  using R = typename SPair<S>::R;
  static constexpr int NT = TX * TY, RN = Ring<TX, TY>::N, CELLS = Ring<TX, TY>::CELLS;
  static constexpr bool BOXED = BOX && kStaged<S, PART>;
  // window planes (the predicted split reads the phase field of every
  // destination, planes z - 1 .. z + 1, after the plane barrier)
  static constexpr int WIN = (kStaged<S, PART> && !SDP) ? 2 : 4;
  static constexpr size_t PHI = (sizeof(C) * WIN * CELLS + 15) / 16 * 16;
  static constexpr int D = kDepth<S, PART>;
  static constexpr size_t OWN = !kStaged<S, PART> ? 0
                                : BOXED          ? sizeof(R) * D * Q * LeanBox<TX, TY>::ELEMS
                                                 : sizeof(R) * D * Q * NT;
  static constexpr size_t RING = (kStaged<S, PART> && !BOXED) ? sizeof(R) * 2 * Q * RN : 0;
  static constexpr size_t SIDE = !PART ? 0
                                 : BOXED ? size_t(D) * (2 * LeanBox<TX, TY>::FB + sizeof(C) * LeanBox<TX, TY>::ELEMS)
                                         : (sizeof(SideRec<C>) * (D * NT + 2 * RN) + 15) / 16 * 16;
  // predicted split: each own / ring cell's phase field of the last step, copied with its pulls
  static constexpr size_t SPL = SDP ? (4 * (D * NT + 2 * RN) + 15) / 16 * 16 : 0;
  // the plane's split barrier; with boxes also FULL[D] and EMPTY[D]
  static constexpr size_t BAR = BOXED ? 8 * (1 + 2 * D + 1) : 16;
  static constexpr size_t BYTES = PHI + OWN + RING + SIDE + SPL + BAR;
  static_assert(PHI % 16 == 0 && OWN % 16 == 0 && RING % 16 == 0 && SIDE % 16 == 0, "stage alignment");
  static __device__ __forceinline__ C (*phi(unsigned char* base))[CELLS] {
    return reinterpret_cast<C(*)[CELLS]>(base);
  }
  static __device__ __forceinline__ R* stage(unsigned char* base) {
    return kStaged<S, PART> ? reinterpret_cast<R*>(base + PHI) : nullptr;
  }
  static __device__ __forceinline__ SideRec<C>* side(unsigned char* base) {
    return PART ? reinterpret_cast<SideRec<C>*>(base + PHI + OWN + RING) : nullptr;
  }
  static __device__ __forceinline__ float* spl(unsigned char* base) {
    return SDP ? reinterpret_cast<float*>(base + PHI + OWN + RING + SIDE) : nullptr;
  }
  static __device__ __forceinline__ unsigned long long* bar(unsigned char* base) {
    return reinterpret_cast<unsigned long long*>(base + PHI + OWN + RING + SIDE + SPL);
  }
  static __device__ __forceinline__ unsigned long long* full(unsigned char* base) { return bar(base) + 1; }
  static __device__ __forceinline__ unsigned long long* empty(unsigned char* base) { return bar(base) + 1 + D; }
  // thread 0 sets up the barriers for the CTA's threads; the caller then syncs
  static __device__ __forceinline__ void init(unsigned char* base) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      mbar_init(bar(base), TX * TY);
      if constexpr (BOXED)
        for (int q = 0; q < 2 * D; ++q) mbar_init(bar(base) + 1 + q, TX * TY);
    }
  }
};

// Barrier phases a CTA has gone through (kept across the columns a
// persistent CTA marches): the plane barrier's parity and, per stage slot,
// the parity of the next FULL / EMPTY phase (bit q)
struct LeanSync {
  unsigned bar = 0, full = 0, empty = 0;
};

// One column march: cells [x0, x0+TX) x [y0, y0+TY) x [z0, zend) of one box.
// SD: the stored pairs are sum / difference pairs (16-bit storage).
template <typename S, int TX, int TY, bool PART, bool SD = false, bool SDP = false, bool BOX = false>
__device__ __forceinline__ void lean_column(const S* __restrict__ A, S* __restrict__ B, const Geom& g,
                                            const LeanConst<typename Store<S>::C>& K, int x0, int y0, int z0,
                                            int zend, unsigned long long* err, int64_t step,
                                            const LeanPart<typename Store<S>::C>& PT,
                                            typename Store<S>::C (*sphi)[Ring<TX, TY>::CELLS],
                                            typename SPair<S>::R* stage, SideRec<typename Store<S>::C>* side,
                                            unsigned long long* bar,
                                            LeanSync& sy, float* spl = nullptr,
                                            const float* __restrict__ split_in = nullptr,
                                            float* __restrict__ split_out = nullptr) {
  using C = typename Store<S>::C;
  constexpr int NT = TX * TY;
  using R = Ring<TX, TY>;
  static_assert(!SD || sizeof(typename SPair<S>::R) == 4, "sum / difference pairs: 16-bit storage");
  static_assert(!SDP || (SD && !PART), "predicted split: sum / difference pairs without spheres");
  const bool parts = PART && PT.fnew != nullptr;  // a box of the ensemble may have no spheres
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const bool active = (x0 + tx < g.nx) && (y0 + ty < g.ny);
  const int x = wrap0(x0 + tx, g.nx), y = wrap0(y0 + ty, g.ny);
  const int own = (ty + 1) * R::RX + (tx + 1);
  // ring cell of this thread (threads 0 .. N-1)
  int rx = 0, ry = 0;
  const bool ringer = tid < R::N;
  if (tid < R::RX) { rx = tid; ry = 0; }
  else if (tid < 2 * R::RX) { rx = tid - R::RX; ry = R::RY - 1; }
  else if (tid < 2 * R::RX + TY) { rx = 0; ry = 1 + tid - 2 * R::RX; }
  else { rx = R::RX - 1; ry = 1 + tid - 2 * R::RX - TY; }
  const int rxg = wrap0(x0 + rx - 1, g.nx), ryg = wrap0(y0 + ry - 1, g.ny);
  const int rslot = ry * R::RX + rx;

  using SR = typename SPair<S>::R;
  constexpr int RN = R::N;
  constexpr bool STAGED = kStaged<S, PART>;
  constexpr bool BOXED = LeanSmem<S, TX, TY, PART, SDP, BOX>::BOXED;
  constexpr int D = kDepth<S, PART>;
  constexpr bool ASYNC = STAGED || PART;  // copy groups in flight
  constexpr bool SPLIT_STORE = !PART;  // see the stores below
  constexpr int WM = LeanSmem<S, TX, TY, PART, SDP, BOX>::WIN - 1;  // window slot of plane p: p & WM
  SR* const ring_stage = (STAGED && !BOXED) ? stage + D * Q * NT : nullptr;
  SideRec<C>* const side_ring = PART ? side + D * NT : nullptr;
  const Planes<const S> Ap{A, 2 * g.n};
  const Planes<S> Bp{B, 2 * g.n};

  // slots of plane p (p >= z0 - 1): own cells D deep, ring cells 2 deep
  // (the own slot q of a plane is passed along: plane z0 - 1 + k has slot
  // k % D, and the march advances it by one per plane without a division)
  auto ring_q = [&](int p) { return (p - z0 + 1) & 1; };
  auto own_slot = [&](int q) { return stage + q * (Q * NT) + tid; };
  auto ring_slot = [&](int p) { return ring_stage + ring_q(p) * (Q * RN) + tid; };

  // Boxes: the slot of plane p holds Q direction boxes of LeanBox::ELEMS
  // pairs; the own / ring cell's pull of direction l is at its base minus e_lx
  using BX = LeanBox<TX, TY>;
  const int obase = (ty + 1) * BX::BW + tx + 4, rbase = ry * BX::BW + rx + 3;
  auto box_slot = [&](int q) { return stage + q * (Q * BX::ELEMS); };
  unsigned long long* const fullb = bar + 1;
  unsigned long long* const emptyb = bar + 1 + D;
  // this thread's granule position: copier threads are the last COPIERS of
  // the CTA (the ring cells sit on the first threads); copier k takes box
  // row r, granule c of the directions of parity grp
  const int ci = tid - (NT - BX::COPIERS);
  const bool copier = BOXED && ci >= 0;
  const int cgrp = ci >= BX::POS ? 1 : 0, cpos = ci - cgrp * BX::POS;
  const int crow = cpos / BX::GR, ccol = cpos - crow * BX::GR;
  // first cell of the granule in its plane for e_ly = +1, 0, -1: row
  // y0 - 1 - e_ly + crow, column x0 - 4 + 4 ccol (periodic; nx % 4 == 0 keeps
  // a granule inside one row)
  unsigned cyx[3] = {0, 0, 0};
  // particle variant, group 0: the flag granule of this copier (array fnew /
  // fold, its first cell in the plane, its place in the flag box)
  unsigned fyx = 0;
  int fdst = -1;
  if constexpr (BOXED) {
    if (copier) {
      const int cxg = wrap0(x0 - 4 + 4 * ccol, g.nx);
#pragma unroll
      for (int k = 0; k < 3; ++k) cyx[k] = unsigned(wrap0(y0 - 1 - (1 - k) + crow, g.ny) * g.nx + cxg);  // k = 1 - e_ly
      if (PART && cgrp == 0 && cpos < BX::FPOS) {
        const int arr = cpos / (BX::ROWS * BX::FGR), rem = cpos - arr * (BX::ROWS * BX::FGR);
        const int frow = rem / BX::FGR, fgr = rem - frow * BX::FGR;
        fyx = unsigned(wrap0(y0 - 1 + frow, g.ny) * g.nx + wrap0(x0 - 16 + 16 * fgr, g.nx));
        fdst = arr * BX::FB + frow * BX::FBW + 16 * fgr;
      }
    }
  }
  // particle boxes of slot q: flags [2][FB] bytes (this step, previous step),
  // then the side phase field [ELEMS]
  unsigned char* const fbox = (PART && BOXED) ? reinterpret_cast<unsigned char*>(side) : nullptr;
  C* const pbox = (PART && BOXED) ? reinterpret_cast<C*>(fbox + D * 2 * BX::FB) : nullptr;
  const int ofb = (ty + 1) * BX::FBW + tx + 16, rfb = ry * BX::FBW + rx + 15;  // own / ring cell's flag byte
  const unsigned plane_cells = unsigned(g.nx) * unsigned(g.ny);
  // the copies of plane p: direction boxes of one parity, one granule each
  auto issue_boxes = [&](int p, int q) {
    SR* const dst = box_slot(q) + crow * BX::BW + 4 * ccol;
    unsigned zo[3];  // plane offsets for e_lz = +1, 0, -1
#pragma unroll
    for (int k = 0; k < 3; ++k) zo[k] = unsigned(wrap_plane(p - (1 - k), g.nz)) * plane_cells;
    auto one = [&](auto lc) {
      constexpr int l = decltype(lc)::value;
      const unsigned cell = zo[1 - ez(l)] + cyx[1 - ey(l)];
      cp_async16(dst + l * BX::ELEMS, Ap.at(l, int(cell)));
    };
    if (cgrp == 0) {
      unroll_even(one);
    } else {
      unroll_odd(one);
    }
    if constexpr (PART) {
      if (parts) {
        if (cgrp == 1)
          cp_async16(pbox + q * BX::ELEMS + crow * BX::BW + 4 * ccol, PT.phi + size_t(zo[1] + cyx[1]));
        else if (fdst >= 0)
          cp_async16(fbox + q * 2 * BX::FB + fdst, (fdst >= BX::FB ? PT.fold : PT.fnew) + size_t(zo[1] + fyx));
      }
    }
  };

  // Start plane p: 16-bit storage copies the pulls of the own and the ring
  // cell into the stage; with spheres, the flag words and the side phase
  // field of both cells are copied too (all in one copy group).
  auto issue = [&](int p, int q) {
    const int zz = wrap_plane(p, g.nz);
    if constexpr (PART && !BOXED) {
      if (parts) {
        // unsigned cell offsets: one 32 x 32 -> 64-bit multiply-add per address
        const unsigned co = unsigned(x) + unsigned(g.nx) * (unsigned(y) + unsigned(g.ny) * unsigned(zz));
        SideRec<C>* so = side + q * NT + tid;
        cp_async4(&so->fnew_w, PT.fnew + size_t(co & ~3u));
        cp_async4(&so->fold_w, PT.fold + size_t(co & ~3u));
        cp_async_c(&so->phi, PT.phi + size_t(co));
        if (ringer) {
          const unsigned cr = unsigned(rxg) + unsigned(g.nx) * (unsigned(ryg) + unsigned(g.ny) * unsigned(zz));
          SideRec<C>* sr = side_ring + ring_q(p) * RN + tid;
          cp_async4(&sr->fnew_w, PT.fnew + size_t(cr & ~3u));
          cp_async4(&sr->fold_w, PT.fold + size_t(cr & ~3u));
          cp_async_c(&sr->phi, PT.phi + size_t(cr));
        }
      }
    }
    if constexpr (BOXED) {
      if (copier) issue_boxes(p, q);
    } else if constexpr (STAGED) {
      PullIdx P;
      pull_idx(g, x, y, zz, P);
      pull_async<S>(A, g.n, P, own_slot(q), NT);
      if (ringer) {
        pull_idx(g, rxg, ryg, zz, P);
        pull_async<S>(A, g.n, P, ring_slot(p), RN);
      }
    }
    if constexpr (SDP) {  // the phase field the pulled pairs were encoded against
      const unsigned co = unsigned(x) + unsigned(g.nx) * (unsigned(y) + unsigned(g.ny) * unsigned(zz));
      cp_async4(spl + q * NT + tid, split_in + size_t(co));
      if (ringer) {
        const unsigned cr = unsigned(rxg) + unsigned(g.nx) * (unsigned(ryg) + unsigned(g.ny) * unsigned(zz));
        cp_async4(spl + D * NT + ring_q(p) * RN + tid, split_in + size_t(cr));
      }
    }
    if constexpr (BOXED) mbar_arrive_cp_async(fullb + q);
    else if constexpr (ASYNC) cp_async_commit();
  };
  auto settle = [&]() {  // every copy group but the newest has landed
    if constexpr (ASYNC && !BOXED) cp_async_wait<1>();
  };
  // boxes: every thread's copies of plane p have landed
  auto full_wait = [&](int q) {
    if constexpr (BOXED) {
      if (!mbar_wait(fullb + q, (sy.full >> q) & 1u)) raise_error(err, LBX_DEV_WAIT_TIMEOUT, step, -2);
      sy.full ^= 1u << q;
    }
  };
  // boxes: this thread has read plane p for the last time / every thread has
  // (the round of the slot this thread arrived at last)
  auto empty_arrive = [&](int q) {
    if constexpr (BOXED) {
      mbar_arrive(emptyb + q);
      sy.empty ^= 1u << q;
    }
  };
  auto empty_wait = [&](int q) {
    if constexpr (BOXED) {
      if (!mbar_wait(emptyb + q, ((sy.empty >> q) & 1u) ^ 1u)) raise_error(err, LBX_DEV_WAIT_TIMEOUT, step, -3);
    }
  };
  // flags (this step, previous step) of a cell from its side record
  auto flags_of = [&](const SideRec<C>* r, int cell, int8_t& fn, int8_t& fo) {
    const int sh = 8 * (cell & 3);
    fn = int8_t((r->fnew_w >> sh) & 255u);
    fo = int8_t((r->fold_w >> sh) & 255u);
  };

  // Phase field (and, for the own cell, the clamped densities) of cell
  // (cx, cy, zz).  Fluid in both steps: pulled densities (16-bit storage sums
  // the pairs its copies brought into the stage, wider types pull here).
  // With spheres, otherwise: a new fluid cell takes the fill kernel's
  // densities, a surface cell the wetting kernel's phase field (both kernels
  // store (rR - rB) / (rR + rB) of the densities they write), and every other
  // solid cell densities 0 (init_rho*_CG's MINDENS).
  // side(cell, fn, fo) gives the cell's flags, side_phi() its side phase field
  auto cell_phase = [&](int cx, int cy, int zz, bool check, bool is_own, auto&& at, auto&& side, auto&& side_phi,
                        C& rR, C& rB, C split) -> C {
    const int cell = cx + g.nx * (cy + g.ny * zz);
    if constexpr (PART) {
      if (parts) {
        int8_t fn, fo;
        side(cell, fn, fo);
        if (fn != LBX_FLUID_FLUID || fo != LBX_FLUID_FLUID) {
          rR = C(0);
          rB = C(0);
          if (fn == LBX_FLUID_SPHERELIST) return side_phi();
          if (fn == LBX_FLUID_FLUID) {  // new fluid cell
            if (is_own) {
              rR = PT.rhoR[2 * size_t(unsigned(cell))];  // interleaved densities
              rB = PT.rhoB[2 * size_t(unsigned(cell))];
            }
            return side_phi();
          }
          return phase_of(rR, rB);
        }
      }
    }
    if constexpr (STAGED) {
      stage_rho<S, C, SD, SDP>(at, K, rR, rB, split);
    } else {
      PullIdx P;
      pull_idx(g, cx, cy, zz, P);
      pull_rho<S, C>(A, g.n, P, K, rR, rB);
    }
    if (check && (rR < C(-10) || rR > C(10) || rB < C(-10) || rB > C(10)))
      raise_error(err, LBX_DEV_RHO_RANGE, step, cell);
    rR = clamp0(rR);
    rB = clamp0(rB);
    return phase_of(rR, rB);
  };

  // phase field of plane p (own cell and ring cell) into its window slot
  auto phase_plane = [&](int p, int q, C& rRo, C& rBo) {
    const int zz = wrap_plane(p, g.nz);
    const bool owned = active && p >= z0 && p < zend;
    const SideRec<C>* so = (PART && !BOXED) ? side + q * NT + tid : nullptr;
    const SR* const ob = BOXED ? box_slot(q) + obase : (STAGED ? own_slot(q) : nullptr);
    auto own_at = [&](int l) -> SR {
      if constexpr (BOXED) return ob[l * BX::ELEMS - ex(l)];
      else return ob[l * NT];
    };
    auto own_side = [&](int cell, int8_t& fn, int8_t& fo) {
      if constexpr (BOXED) {
        fn = int8_t(fbox[q * 2 * BX::FB + ofb]);
        fo = int8_t(fbox[q * 2 * BX::FB + BX::FB + ofb]);
      } else {
        flags_of(so, cell, fn, fo);
      }
    };
    auto own_sphi = [&]() -> C {
      if constexpr (BOXED) return pbox[q * BX::ELEMS + obase];
      else return so->phi;
    };
    sphi[p & WM][own] = cell_phase(x, y, zz, owned, true, own_at, own_side, own_sphi, rRo, rBo,
                                   SDP ? C(spl[q * NT + tid]) : C(0));
    if (ringer) {
      C qR, qB;
      const SideRec<C>* sr = (PART && !BOXED) ? side_ring + ring_q(p) * RN + tid : nullptr;
      const SR* const rb = BOXED ? box_slot(q) + rbase : (STAGED ? ring_slot(p) : nullptr);
      auto ring_at = [&](int l) -> SR {
        if constexpr (BOXED) return rb[l * BX::ELEMS - ex(l)];
        else return rb[l * RN];
      };
      auto ring_side = [&](int cell, int8_t& fn, int8_t& fo) {
        if constexpr (BOXED) {
          fn = int8_t(fbox[q * 2 * BX::FB + rfb]);
          fo = int8_t(fbox[q * 2 * BX::FB + BX::FB + rfb]);
        } else {
          flags_of(sr, cell, fn, fo);
        }
      };
      auto ring_sphi = [&]() -> C {
        if constexpr (BOXED) return pbox[q * BX::ELEMS + rbase];
        else return sr->phi;
      };
      sphi[p & WM][rslot] = cell_phase(rxg, ryg, zz, false, false, ring_at, ring_side, ring_sphi, qR, qB,
                                       SDP ? C(spl[D * NT + ring_q(p) * RN + tid]) : C(0));
    }
  };

  C rRn, rBn, rRc, rBc;
  issue(z0 - 1, 0);
  issue(z0, 1);
  settle();
  full_wait(0);
  phase_plane(z0 - 1, 0, rRc, rBc);
  issue(z0 + 1, 2 % D);
  settle();
  full_wait(1);
  phase_plane(z0, 1, rRn, rBn);
  __syncthreads();  // planes z0-1 and z0 of the window
  PlaneGrad<C> gm{}, g0{};
  if constexpr (STAGED) {
    if (active) {
      gm = plane_grad<C, R::RX>(sphi[(z0 - 1) & WM], own);
      g0 = plane_grad<C, R::RX>(sphi[z0 & WM], own);
    }
    __syncthreads();  // the slot of plane z0-1 is rewritten in the first iteration
  }
  int qz = 1;  // own slot of plane z
  for (int z = z0; z < zend; ++z) {
    rRc = rRn;
    rBc = rBn;
    const int q1 = qz == D - 1 ? 0 : qz + 1;  // plane z+1
    const int q2 = q1 == D - 1 ? 0 : q1 + 1;  // plane z+2, the slot of plane z-1
    // plane z+2 is copied while z+1 is summed and z collided; the copies
    // into the slots of plane z-1 start after this thread's last read of them
    // (boxes: after every thread's; plane z0-1 was read in the prologue only)
    // Boxes: copy group 0 issues its granules of plane z+2 here, group 1
    // after its phase sums, so that the two bursts of 16-byte copies do not
    // fill the memory-instruction queue together (FP16 128^3: 82.6 us against
    // 88.8 with every copy here, 92.8 with every copy after the BGK half)
    const bool late = BOXED && cgrp == 1;
    if (z + 2 <= zend) {
      if (z > z0) empty_wait(q2);
      if (!late) issue(z + 2, q2);
    } else if constexpr (ASYNC && !BOXED) {
      cp_async_commit();  // one group per iteration
    }
    settle();
    full_wait(q1);
    phase_plane(z + 1, q1, rRn, rBn);
    if (late && z + 2 <= zend) issue(z + 2, q2);
    mbar_arrive(bar);
    // Window reads: with staged pulls, plane z+1 after the wait below (its
    // other slot, plane z+2, is written in the next iteration, after every
    // thread has arrived at this plane's barrier, i.e. finished these reads);
    // otherwise planes z-1 and z before the wait (written before the previous
    // plane's barrier, rewritten only after this one) and z+1 after it.
    const int cell = x + g.nx * (y + g.ny * z);
    bool collide = true;
    C px = 0, py = 0, pz = 0;
    Relaxed<C> rx;
    if (active) {
      if constexpr (PART) {
        if (parts) {
          int8_t fn, fo;
          if constexpr (BOXED) {
            fn = int8_t(fbox[qz * 2 * BX::FB + ofb]);
            fo = int8_t(fbox[qz * 2 * BX::FB + BX::FB + ofb]);
          } else {
            flags_of(side + qz * NT + tid, cell, fn, fo);
          }
          // a solid cell keeps the plain pull (see below); a cell that
          // turns fluid pulls the populations make_fluid wrote into the
          // slots it pulls from
          collide = fn == LBX_FLUID_FLUID;
        }
      }
    }
    // Stored pairs of this cell: the pull (in the stage since two
    // iterations, or issued here).
    const SR* const zb = BOXED ? box_slot(qz) + obase : nullptr;
    auto pulled = [&](int l) -> SR {
      if constexpr (BOXED) return zb[l * BX::ELEMS - ex(l)];
      else if constexpr (STAGED) return own_slot(qz)[l * NT];
      else return SPair<S>::ldr(Ap.at(l, pull_one(g, x, y, z, l)));
    };
    if (active && collide) {
      // the colour gradient from planes z-1 and z (synchronous pulls only),
      // then the BGK half
      if constexpr (!STAGED) {
        const C* pm = sphi[(z + 3) & 3];
        const C* p0 = sphi[z & 3];
#pragma unroll
        for (int l = 1; l < Q27; ++l) {
          const int dx = ex27(l), dy = ey27(l), dz = ez27(l);
          if (dz > 0) continue;
          const C* pl = dz < 0 ? pm : p0;
          const C ps = pl[own + dy * R::RX + dx];
          const C a = K.a27[wclass27(l)];
          if (dx) px = fm(dx > 0 ? a : -a, ps, px);
          if (dy) py = fm(dy > 0 ? a : -a, ps, py);
          if (dz) pz = fm(dz > 0 ? a : -a, ps, pz);
        }
      }
      C Ssum[Q];
#pragma unroll
      for (int l = 0; l < Q; ++l) Ssum[l] = SD ? SPair<S>::first(pulled(l)) : SPair<S>::sum(pulled(l));
      rx = relax_sums(K, Ssum, rRc, rBc, Store<S>::shifted);
    }
    if (!mbar_wait(bar, sy.bar)) raise_error(err, LBX_DEV_WAIT_TIMEOUT, step, -1);
    sy.bar ^= 1u;
    const C* const win[3] = {sphi[(z - 1) & WM], sphi[z & WM], sphi[(z + 1) & WM]};  // planes z - 1 .. z + 1
    (void)win;
    if (active) {
      // A solid cell stores its streamed populations as pulled.  The
      // reference's push leaves a stale value behind a spheredead source
      // instead; no fluid cell, force or moment ever reads a solid cell's
      // populations (a fluid cell pulls from a solid one only along a link
      // the bounce-back rewrote, and a cell that turns fluid is refilled), so
      // only raw population dumps of solid cells differ.
      P2<C> gp[Q];
      bool done = false;
      auto store_all = [&](const P2<C>* v) {
#pragma unroll
        for (int l = 0; l < Q; ++l) SPair<S>::st(Bp.at(l, cell), v[l]);
      };
      if constexpr (STAGED) {
        const PlaneGrad<C> gpl = plane_grad<C, R::RX>(sphi[(z + 1) & WM], own);
        if (collide) {
          const C H0 = C(1) / C(3), H1 = C(1) / C(12), HALF = C(0.5);  // W / 2
          px = fm(H0, g0.gx, H1 * (gm.gx + gpl.gx));
          py = fm(H0, g0.gy, H1 * (gm.gy + gpl.gy));
          pz = HALF * (gpl.m - gm.m);
        }
        gm = g0;
        g0 = gpl;
      }
      if (collide) {
        if constexpr (!STAGED) {  // plane z+1 of the colour gradient
          const C* ppl = sphi[(z + 1) & 3];
#pragma unroll
          for (int l = 1; l < Q27; ++l) {
            const int dx = ex27(l), dy = ey27(l), dz = ez27(l);
            if (dz <= 0) continue;
            const C ps = ppl[own + dy * R::RX + dx];
            const C a = K.a27[wclass27(l)];
            if (dx) px = fm(dx > 0 ? a : -a, ps, px);
            if (dy) py = fm(dy > 0 ? a : -a, ps, py);
            pz = fm(a, ps, pz);
          }
        }
        done = recolour_sums<C, SD, SDP, R::RX>(K, rx, rRc, rBc, px, py, pz, Store<S>::shifted, gp, win, own);
        // stored on each path by itself: one set of values per path, no
        // register copies to merge the two (FP16 128^3: 806 -> 718
        // instructions per cell with the other changes of the box staging).
        // With spheres one store after the merge measured faster (838
        // against 856 instructions per cell, 111 against 114 us at 128^3 with
        // 160 spheres; without the new-cell case 827 against 817 and 110 us
        // both, but 691 against 701 us at 256^3 with 1280 spheres), and the
        // persistent multi-box kernel would spill.
        if constexpr (SPLIT_STORE)
          if (done) store_all(gp);
      }
      if (!done) {
#pragma unroll
        for (int l = 0; l < Q; ++l) gp[l] = SPair<S>::cvt(pulled(l));
        if constexpr (SDP) {  // (total, E) -> (total, R - B) with this cell's split of the last step
          const C ph = spl[qz * NT + tid];
#pragma unroll
          for (int l = 0; l < Q; ++l) gp[l].y = fm(ph, gp[l].x + K.ssd[0][wclass(l)], gp[l].y);
        }
        if (collide) {
          if constexpr (SD) bgk_components<C, STAGED, true>(K, rx, rRc + rBc, rRc - rBc, Store<S>::shifted, gp);
          else bgk_components<C, STAGED>(K, rx, rRc, rBc, Store<S>::shifted, gp);
        }
        if constexpr (SDP) {  // R - B -> E against the split of each receiving cell
#pragma unroll
          for (int l = 0; l < Q; ++l)
            gp[l].y = fm(-win[1 + ez(l)][own + ey(l) * R::RX + ex(l)], gp[l].x + K.ssd[0][wclass(l)], gp[l].y);
        }
        if constexpr (SPLIT_STORE) store_all(gp);
      }
      if constexpr (!SPLIT_STORE) store_all(gp);
      if constexpr (SDP) split_out[size_t(unsigned(cell))] = sphi[z & WM][own];  // what the receivers decode with
    }
    // boxes: plane z is not read again; its slot takes plane z+3 next iteration
    if (z + 3 <= zend) empty_arrive(qz);
    qz = q1;
  }
  if constexpr (ASYNC) cp_async_wait<0>();  // nothing in flight when the shared memory is reused
}

template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool SDP = false, bool BOX = false>
__global__ void __launch_bounds__(TX* TY, MINB)
    k_cg_lean(const S* __restrict__ A, S* __restrict__ B, Geom g, LeanConst<typename Store<S>::C> K, int zlen,
              unsigned long long* err, int64_t step, LeanPart<typename Store<S>::C> PT,
              const float* __restrict__ split_in, float* __restrict__ split_out, const int4* __restrict__ plan) {
  extern __shared__ __align__(16) unsigned char lean_smem[];
  using M = LeanSmem<S, TX, TY, PART, SDP, BOX>;
  M::init(lean_smem);
  __syncthreads();
  LeanSync sy;
  // the column and z-segment of this CTA: from the grid (equal segments) or
  // from the launch's plan (x0, y0, z0, zend per CTA)
  int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * zlen, z1 = min(z0 + zlen, g.nz);
  if (plan) {
    const int4 w = plan[blockIdx.x];
    x0 = w.x;
    y0 = w.y;
    z0 = w.z;
    z1 = w.w;
  }
  lean_column<S, TX, TY, PART, SD, SDP, BOX>(A, B, g, K, x0, y0, z0, z1, err, step, PT, M::phi(lean_smem),
                                             M::stage(lean_smem), M::side(lean_smem), M::bar(lean_smem), sy,
                                             M::spl(lean_smem), split_in, split_out);
}

// ---------------------------------------------------------------------------
// Several independent boxes in one persistent launch: each CTA takes work
// items (box, column, z-segment) from a table, longest first, and marches
// them like k_cg_lean.  Used by the ensemble of uneven boxes.
// ---------------------------------------------------------------------------
template <typename C>
struct BoxDesc {
  const void* A;
  void* B;
  Geom g;
  LeanPart<C> pt;
  unsigned long long* err;
  int64_t step;
};

struct WorkItem {
  int box, x0, y0, z0, zend;
};

template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool BOX = false>
__global__ void __launch_bounds__(TX* TY, MINB)
    k_cg_lean_multi(const BoxDesc<typename Store<S>::C>* __restrict__ boxes, const WorkItem* __restrict__ work,
                    int nwork, LeanConst<typename Store<S>::C> K) {
  using C = typename Store<S>::C;
  extern __shared__ __align__(16) unsigned char lean_smem[];
  using M = LeanSmem<S, TX, TY, PART, false, BOX>;
  M::init(lean_smem);
  __syncthreads();
  LeanSync sy;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const WorkItem it = work[w];
    const BoxDesc<C> bd = boxes[it.box];
    lean_column<S, TX, TY, PART, SD, false, BOX>((const S*)bd.A, (S*)bd.B, bd.g, K, it.x0, it.y0, it.z0, it.zend,
                                                bd.err, bd.step, bd.pt, M::phi(lean_smem), M::stage(lean_smem),
                                                M::side(lean_smem), M::bar(lean_smem), sy);
    __syncthreads();  // the window and the stage are reused by the next item
  }
}

// ---------------------------------------------------------------------------
// z-segment length of the fluid kernel.  A segment costs two extra planes
// (its halo in z), so segments should be long; neighbouring columns read each
// other's edge cells (the ring) from L2, so the CTAs that run together should
// march neighbouring columns over nearby planes, which many short waves of
// equal segments do.  Segments of 32 planes, or, when that leaves the first
// wave of resident CTAs short, as many equal segments per column as fit in
// one wave.  Measured on B200 (FP16 / FP32 ms per step): 128^3, 4 segments
// of 32: 0.127 / 0.168, against 10 of 13: 0.129 / 0.183, and 2 of 64:
// 0.145 / 0.259; 256^3, segments of 32: 0.81 / 1.19, of 64: 0.81 / 1.27,
// whole columns: 0.93 / 1.34.
static int lean_zlen(const Ctx& c, int tx, int ty, int resident) {
  const long cols = long((c.nx + tx - 1) / tx) * long((c.ny + ty - 1) / ty);
  long segs = (c.nz + 31) / 32;
  if (cols * segs <= resident) segs = std::max(segs, long(resident) / cols);
  segs = std::max(1L, std::min<long>(segs, c.nz));
  return int((c.nz + segs - 1) / segs);
}

// Paired segment plan.  When four equal z-segments per column leave resident
// CTA slots empty and five would need a second wave (128^3 with 32 x 8
// columns: 256 CTAs for 296 slots, so 40 SMs run one CTA and the kernel takes
// as long as two 32-plane segments on the others), some columns are cut into
// one segment of nz/4 planes and four of the rest's quarter, the others into
// four of nz/4, and all long segments are launched before the short ones:
// the scheduler then gives each SM one long and one short segment (at 128^3:
// 37 columns of 32 + 4 x 24 planes, 27 of 4 x 32; 145 long, 148 short).
// Returns the device table (x0, y0, z0, zend per CTA) kept in the context, or
// nullptr when the equal segments are used.
static const int4* paired_plan(Ctx& c, int TX, int TY, int resident, int* n) {
  // the planes marched: the whole box, or a z-slab's own planes
  const int zb = c.zhi > 0 ? c.zlo : 0, nzr = (c.zhi > 0 ? c.zhi : c.nz) - zb;
  const int ncx = (c.nx + TX - 1) / TX, ncy = (c.ny + TY - 1) / TY, cols = ncx * ncy;
  const int b = std::min(cols, std::min(resident / 8, resident - 4 * cols));  // columns cut 1 + 4
  if (nzr < 64 || 4 * cols >= resident || 5 * cols <= resident || b <= 0) return nullptr;
  const int64_t key = ((int64_t(resident) * 4096 + TX * 64 + TY) * 65536 + zb) * 65536 + nzr;
  if (c.lean_plan && c.lean_plan_key == key) {
    *n = c.lean_plan_n;
    return static_cast<const int4*>(c.lean_plan);
  }
  std::vector<int4> lng, sht;
  const int L1 = nzr / 4, rest = nzr - L1;
  for (int col = 0; col < cols; ++col) {
    const int x0 = (col % ncx) * TX, y0 = (col / ncx) * TY;
    const bool cut = (long(col) * b) / cols != (long(col + 1) * b) / cols;  // b columns spread over all
    if (!cut) {
      for (int k = 0; k < 4; ++k) lng.push_back(make_int4(x0, y0, zb + k * nzr / 4, zb + (k + 1) * nzr / 4));
    } else {
      lng.push_back(make_int4(x0, y0, zb, zb + L1));
      for (int k = 0; k < 4; ++k)
        sht.push_back(make_int4(x0, y0, zb + L1 + k * rest / 4, zb + L1 + (k + 1) * rest / 4));
    }
  }
  lng.insert(lng.end(), sht.begin(), sht.end());
  if (c.lean_plan) cudaFree(c.lean_plan);
  c.lean_plan = nullptr;
  if (cudaMalloc(&c.lean_plan, lng.size() * sizeof(int4)) != cudaSuccess) {
    c.lean_plan = nullptr;
    return nullptr;
  }
  cudaMemcpy(c.lean_plan, lng.data(), lng.size() * sizeof(int4), cudaMemcpyHostToDevice);
  c.lean_plan_n = int(lng.size());
  c.lean_plan_key = key;
  *n = c.lean_plan_n;
  return static_cast<const int4*>(c.lean_plan);
}

// Plan of a z-slab (lbx_set_zrange): every column marched over the own planes
// [zlo, zhi) only, in equal segments of at most 32 planes (as many as fill
// the resident CTA slots when there are fewer).  Cached in the context like
// the paired plan.
static const int4* range_plan(Ctx& c, int TX, int TY, int resident, int* n) {
  const int ncx = (c.nx + TX - 1) / TX, ncy = (c.ny + TY - 1) / TY, cols = ncx * ncy;
  const int own = c.zhi - c.zlo;
  long segs = (own + 31) / 32;
  if (long(cols) * segs <= resident) segs = std::max(segs, long(resident) / cols);
  segs = std::max(1L, std::min<long>(segs, own));
  // negative: never a paired plan's key
  const int64_t key = -(1 + int64_t(c.zlo) + 65536 * (int64_t(c.zhi) + 65536 * (int64_t(TY) + 64 * segs)));
  if (c.lean_plan && c.lean_plan_key == key) {
    *n = c.lean_plan_n;
    return static_cast<const int4*>(c.lean_plan);
  }
  std::vector<int4> plan;
  for (long k = 0; k < segs; ++k)
    for (int col = 0; col < cols; ++col)
      plan.push_back(make_int4((col % ncx) * TX, (col / ncx) * TY, c.zlo + int(k * own / segs),
                               c.zlo + int((k + 1) * own / segs)));
  if (c.lean_plan) cudaFree(c.lean_plan);
  c.lean_plan = nullptr;
  if (cudaMalloc(&c.lean_plan, plan.size() * sizeof(int4)) != cudaSuccess) {
    c.lean_plan = nullptr;
    return nullptr;
  }
  cudaMemcpy(c.lean_plan, plan.data(), plan.size() * sizeof(int4), cudaMemcpyHostToDevice);
  c.lean_plan_n = int(plan.size());
  c.lean_plan_key = key;
  *n = c.lean_plan_n;
  return static_cast<const int4*>(c.lean_plan);
}

// Opt a kernel into its dynamic shared memory (beyond the default 48 KB), once
// per device.  Called outside stream capture (the first eager launch, or when
// an ensemble builds its tables).
template <typename K>
static int allow_smem(K* kernel, size_t bytes, unsigned long long& done_mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LBX_ERR_CUDA;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done_mask & bit) return 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) != cudaSuccess)
    return LBX_ERR_CUDA;
  done_mask |= bit;
  return 0;
}

// Opt-in of k_cg_lean's shared memory and its resident CTAs per SM on this
// device (the persistent grid), once per device.
template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool SDP = false, bool BOX = false>
static int prepare_lean(int* resident) {
  static unsigned long long done = 0;
  static int per_sm[64] = {0}, sms[64] = {0};
  using M = LeanSmem<S, TX, TY, PART, SDP, BOX>;
  int rc = allow_smem(k_cg_lean<S, TX, TY, MINB, PART, SD, SDP, BOX>, M::BYTES, done);
  if (rc) return rc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LBX_ERR_CUDA;
  dev &= 63;
  if (!per_sm[dev]) {
    int nb = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_cg_lean<S, TX, TY, MINB, PART, SD, SDP, BOX>, TX * TY,
                                                      M::BYTES) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nb < 1 || nsm < 1)
      return LBX_ERR_CUDA;
    sms[dev] = nsm;
    per_sm[dev] = nb;
  }
  *resident = per_sm[dev] * sms[dev];
  return 0;
}

template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool BOX = false>
static int prepare_lean_multi() {
  static unsigned long long done = 0;
  return allow_smem(k_cg_lean_multi<S, TX, TY, MINB, PART, SD, BOX>, LeanSmem<S, TX, TY, PART, false, BOX>::BYTES,
                    done);
}

// Box copies (16-bit storage): when nx is a multiple of 4 (a 16-byte granule
// then never straddles the periodic x edge) unless switched off
static bool use_boxes(const Ctx& c, bool part = false) {
  return c.lean_copies == 1 && c.nx % (part ? 16 : 4) == 0;
}

template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool SDP = false, bool BOX = false>
static int launch_lean_as(Ctx& c, int zlen_override, LeanPart<typename Store<S>::C> pt) {
  using C = typename Store<S>::C;
  int resident = 0;
  const int rc = prepare_lean<S, TX, TY, MINB, PART, SD, SDP, BOX>(&resident);
  if (rc) return rc;
  const int zlen = zlen_override > 0 ? zlen_override : lean_zlen(c, TX, TY, resident);
  dim3 block(TX, TY, 1);
  dim3 grid((c.nx + TX - 1) / TX, (c.ny + TY - 1) / TY, (c.nz + zlen - 1) / zlen);
  // the paired plan only for the staged 16-bit kernels: FP32 / FP64 re-read
  // their pairs from L2, which neighbouring columns out of step in z defeat
  // (FP32 128^3: 185 us with the plan, 148 us without; FP16 96 against 101)
  int nplan = 0;
  const int4* plan = nullptr;
  if (zlen_override <= 0 && kStaged<S, PART>) plan = paired_plan(c, TX, TY, resident, &nplan);
  if (!plan && c.zhi > 0) {  // a z-slab: only its own planes
    plan = range_plan(c, TX, TY, resident, &nplan);
    if (!plan) return LBX_ERR_ALLOC;
  }
  if (plan) grid = dim3(unsigned(nplan), 1, 1);
  k_cg_lean<S, TX, TY, MINB, PART, SD, SDP, BOX>
      <<<grid, block, LeanSmem<S, TX, TY, PART, SDP, BOX>::BYTES, c.stream>>>(
          (const S*)c.pops[c.cur], (S*)c.pops[1 - c.cur], geom(c), make_lean<C>(c), zlen, c.d_err, c.step + 1, pt,
          SDP ? c.split[c.cur] : nullptr, SDP ? c.split[1 - c.cur] : nullptr, plan);
  return 0;
}

template <typename S, int TX, int TY, int MINB, bool PART, bool SD = false, bool SDP = false>
static int launch_lean(Ctx& c, int zlen_override, LeanPart<typename Store<S>::C> pt) {
  if constexpr (kStaged<S, PART>) {
    if (use_boxes(c, PART)) return launch_lean_as<S, TX, TY, MINB, PART, SD, SDP, true>(c, zlen_override, pt);
  }
  return launch_lean_as<S, TX, TY, MINB, PART, SD, SDP, false>(c, zlen_override, pt);
}

void kt_begin(Ctx& c);
void kt_end(Ctx& c);

// shape: 0 = 32x8 (two CTAs per SM), 1 = 32x16 (one CTA per SM)
int fluid_lean(Ctx& c) {
  int rc = by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    LeanPart<C> none{nullptr, nullptr, nullptr, nullptr, nullptr};
    kt_begin(c);
    int r = 0;
    if constexpr (std::is_same<S, double>::value) {
      r = launch_lean<S, 32, 8, 1, false>(c, c.lean_zlen, none);
    } else if constexpr (std::is_same<S, float>::value) {
      if (c.lean_shape == 1) r = launch_lean<S, 32, 16, 1, false>(c, c.lean_zlen, none);
      else r = launch_lean<S, 32, 8, 2, false>(c, c.lean_zlen, none);
    } else if (c.sdp) {  // sum / predicted-split pairs
      r = launch_lean<S, 32, 8, 2, false, true, true>(c, c.lean_zlen, none);
    } else if (c.sd) {  // sum / difference pairs
      if (c.lean_shape == 1) r = launch_lean<S, 32, 16, 1, false, true>(c, c.lean_zlen, none);
      else r = launch_lean<S, 32, 8, 2, false, true>(c, c.lean_zlen, none);
    } else {
      if (c.lean_shape == 1) r = launch_lean<S, 32, 16, 1, false>(c, c.lean_zlen, none);
      else r = launch_lean<S, 32, 8, 2, false>(c, c.lean_zlen, none);
    }
    kt_end(c);
    return r ? r : launch_status();
  });
  if (!rc) c.cur = 1 - c.cur;
  return rc;
}

// the same step with particle flags (fo: flags of the previous step, fn: of this one)
int fluid_lean_particles(Ctx& c, int fo, int fn) {
  int rc = by_storage(c, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    LeanPart<C> pt{c.flags[fo], c.flags[fn], (C*)c.rho[0], (C*)c.rho[1], (C*)c.phi};
    kt_begin(c);
    int r = 0;
    if constexpr (std::is_same<S, double>::value) r = launch_lean<S, 32, 8, 1, true>(c, c.lean_zlen, pt);
    else if constexpr (std::is_same<S, float>::value) r = launch_lean<S, 32, 8, 2, true>(c, c.lean_zlen, pt);
    else if (c.sd) r = launch_lean<S, 32, 8, 2, true, true>(c, c.lean_zlen, pt);
    else r = launch_lean<S, 32, 8, 2, true>(c, c.lean_zlen, pt);
    kt_end(c);
    return r ? r : launch_status();
  });
  return rc;  // the particle step swaps the buffers after its bounce-back
}

}  // namespace lbx

namespace lbx {

int particles_active(const Ctx& c);

// Build (build_only = 1: returns the number of work items) or launch the
// persistent multi-box kernel of an ensemble for the given buffer parity.
int ensemble_launch(const std::vector<Ctx*>& boxes, int shape, const std::vector<int>& zlen, void* d_desc,
                    void* d_work, int nwork, cudaStream_t stream, int build_only, int parity) {
  if (boxes.empty()) return LBX_ERR_ARG;
  const Ctx& c0 = *boxes[0];
  const int TX = 32, TY = shape == 1 ? 16 : 8;
  // The persistent kernel keeps each work item's box descriptor in
  // registers, which leaves no room for the box copies' per-thread state
  // without spills (measured: 8-16 bytes per thread), so it stages its 16-bit
  // pulls one copy per pull (BOX = false).
  return by_storage(c0, [&](auto* tag) -> int {
    using S = std::remove_pointer_t<decltype(tag)>;
    using C = typename Store<S>::C;
    if (build_only) {
      std::vector<BoxDesc<C>> desc(boxes.size());
      std::vector<WorkItem> work;
      for (size_t b = 0; b < boxes.size(); ++b) {
        const Ctx& c = *boxes[b];
        BoxDesc<C>& d = desc[b];
        d.A = c.pops[parity];
        d.B = c.pops[1 - parity];
        d.g = geom(c);
        const bool parts = particles_active(c) != 0;
        d.pt = LeanPart<C>{parts ? c.flags[parity] : nullptr, parts ? c.flags[1 - parity] : nullptr,
                           parts ? (C*)c.rho[0] : nullptr, parts ? (C*)c.rho[1] : nullptr,
                           parts ? (C*)c.phi : nullptr};
        d.err = c.d_err;
        d.step = c.step + 1;
        const int zl = std::max(1, zlen[b]);
        for (int z0 = 0; z0 < c.nz; z0 += zl)
          for (int y0 = 0; y0 < c.ny; y0 += TY)
            for (int x0 = 0; x0 < c.nx; x0 += TX) work.push_back(WorkItem{int(b), x0, y0, z0, std::min(z0 + zl, c.nz)});
      }
      std::stable_sort(work.begin(), work.end(),
                       [](const WorkItem& a, const WorkItem& b) { return (a.zend - a.z0) > (b.zend - b.z0); });
      if (desc.size() * sizeof(BoxDesc<C>) > 512 * desc.size()) return LBX_ERR_STATE;
      // shared-memory opt-in of every variant, before any capture
      int rp = 0;
      if constexpr (std::is_same<S, double>::value) {
        rp = prepare_lean_multi<S, 32, 8, 1, true>();
      } else if constexpr (std::is_same<S, float>::value) {
        rp = prepare_lean_multi<S, 32, 16, 1, true>();
        if (!rp) rp = prepare_lean_multi<S, 32, 8, 2, true>();
      } else if (c0.sd) {
        rp = prepare_lean_multi<S, 32, 16, 1, true, true>();
        if (!rp) rp = prepare_lean_multi<S, 32, 8, 2, true, true>();
      } else {
        rp = prepare_lean_multi<S, 32, 16, 1, true>();
        if (!rp) rp = prepare_lean_multi<S, 32, 8, 2, true>();
      }
      if (rp) return rp;
      if (cudaMemcpy(d_desc, desc.data(), desc.size() * sizeof(BoxDesc<C>), cudaMemcpyHostToDevice) != cudaSuccess)
        return LBX_ERR_CUDA;
      if (cudaMemcpy(d_work, work.data(), work.size() * sizeof(WorkItem), cudaMemcpyHostToDevice) != cudaSuccess)
        return LBX_ERR_CUDA;
      return int(work.size());
    }
    const LeanConst<C> K = make_lean<C>(c0);
    const auto* D = (const BoxDesc<C>*)d_desc;
    const auto* W = (const WorkItem*)d_work;
    if constexpr (std::is_same<S, double>::value) {
      int grid = std::min(nwork, 148);
      k_cg_lean_multi<S, 32, 8, 1, true><<<grid, dim3(32, 8), LeanSmem<S, 32, 8, true>::BYTES, stream>>>(D, W, nwork, K);
    } else if constexpr (std::is_same<S, float>::value) {
      if (shape == 1)
        k_cg_lean_multi<S, 32, 16, 1, true><<<std::min(nwork, 148), dim3(32, 16), LeanSmem<S, 32, 16, true>::BYTES,
                                                stream>>>(D, W, nwork, K);
      else
        k_cg_lean_multi<S, 32, 8, 2, true><<<std::min(nwork, 296), dim3(32, 8), LeanSmem<S, 32, 8, true>::BYTES,
                                               stream>>>(D, W, nwork, K);
    } else {
      auto go = [&](auto sd_tag) {
        constexpr bool SDV = decltype(sd_tag)::value;
        if (shape == 1)
          k_cg_lean_multi<S, 32, 16, 1, true, SDV>
              <<<std::min(nwork, 148), dim3(32, 16), LeanSmem<S, 32, 16, true>::BYTES, stream>>>(D, W, nwork, K);
        else
          k_cg_lean_multi<S, 32, 8, 2, true, SDV>
              <<<std::min(nwork, 296), dim3(32, 8), LeanSmem<S, 32, 8, true>::BYTES, stream>>>(D, W, nwork, K);
      };
      if (c0.sd) go(std::true_type{});
      else go(std::false_type{});
    }
    return launch_status();
  });
}

}  // namespace lbx
