// lbx_closure.h — the learned pair closure shared by its training/inference
// kernels (lbx_closure.cu) and the particle step (lbx_particles.cu):
// network dimensions, the weight-blob layout, the warp-level forward pass and
// the lattice-fixed pair frame.
#pragma once
#include <cuda_runtime.h>

#include "../../include/lbx.h"

namespace lbx {
constexpr int DIN = 13, H = 64, DOUT = 12;

// parameter offsets in the flat weight blob
struct MlpLayout {
  static constexpr int W0 = 0, B0 = W0 + H * DIN, W1 = B0 + H, B1 = W1 + H * H, W2 = B1 + H, B2 = W2 + H * H,
                       W3 = B2 + H, B3 = W3 + DOUT * H, NPARAM = B3 + DOUT;
  static constexpr int XMU = NPARAM, XSD = XMU + DIN, YMU = XSD + DIN, YSD = YMU + DOUT, TOTAL = YSD + DOUT;
};
static_assert(MlpLayout::TOTAL == LBX_CLOSURE_NWEIGHTS, "weight blob layout");

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Shared-memory copy of the blob for inference with the 64-wide matrices
// transposed (W[k][o]), so that lane o reads consecutive words.
__device__ inline void load_infer_weights(const float* __restrict__ Wg, float* W) {
  using L = MlpLayout;
  for (int i = threadIdx.x; i < L::TOTAL; i += blockDim.x) {
    float v = Wg[i];
    int j = i;
    if (i >= L::W1 && i < L::B1) { int o = (i - L::W1) / H, k = (i - L::W1) % H; j = L::W1 + k * H + o; }
    else if (i >= L::W2 && i < L::B2) { int o = (i - L::W2) / H, k = (i - L::W2) % H; j = L::W2 + k * H + o; }
    else if (i >= L::W3 && i < L::B3) { int o = (i - L::W3) / H, k = (i - L::W3) % H; j = L::W3 + k * DOUT + o; }
    W[j] = v;
  }
}

__device__ inline void mlp_warp(const float* W, const float x_raw[DIN], float y_raw[DOUT], float* buf /* 2*H */) {
  using L = MlpLayout;
  const int lane = threadIdx.x & 31;
  // standardised input, broadcast through the warp buffer
  if (lane < DIN) buf[lane] = (x_raw[lane] - W[L::XMU + lane]) / W[L::XSD + lane];
  __syncwarp();
  float h0[2];
  for (int r = 0; r < 2; ++r) {
    int o = lane + 32 * r;
    float s = W[L::B0 + o];
    for (int k = 0; k < DIN; ++k) s = fmaf(buf[k], W[L::W0 + o * DIN + k], s);
    h0[r] = silu(s);
  }
  __syncwarp();
  buf[lane] = h0[0];
  buf[lane + 32] = h0[1];
  __syncwarp();
  const int Wl[2] = {L::W1, L::W2}, Bl[2] = {L::B1, L::B2};
  for (int layer = 0; layer < 2; ++layer) {
    float h[2];
    for (int r = 0; r < 2; ++r) {
      int o = lane + 32 * r;
      float s = W[Bl[layer] + o];
      for (int k = 0; k < H; ++k) s = fmaf(buf[k], W[Wl[layer] + k * H + o], s);
      h[r] = silu(s);
    }
    __syncwarp();
    buf[lane] = h[0];
    buf[lane + 32] = h[1];
    __syncwarp();
  }
  float yl = 0.f;
  if (lane < DOUT) {
    float s = W[L::B3 + lane];
    for (int k = 0; k < H; ++k) s = fmaf(buf[k], W[L::W3 + k * DOUT + lane], s);
    yl = s * W[L::YSD + lane] + W[L::YMU + lane];
  }
  for (int o = 0; o < DOUT; ++o) y_raw[o] = __shfl_sync(0xffffffffu, yl, o);
  __syncwarp();
}

// ---------------------------------------------------------------------------
// pair frame and features (shared with the host-side data generation)
// ---------------------------------------------------------------------------
__host__ __device__ inline void pair_frame(const double n[3], double t1[3], double t2[3]) {
  double ax = fabs(n[0]), ay = fabs(n[1]), az = fabs(n[2]);
  double e[3] = {0, 0, 0};
  if (ax <= ay && ax <= az) e[0] = 1; else if (ay <= az) e[1] = 1; else e[2] = 1;
  double c[3] = {n[1] * e[2] - n[2] * e[1], n[2] * e[0] - n[0] * e[2], n[0] * e[1] - n[1] * e[0]};
  double m = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int d = 0; d < 3; ++d) t1[d] = c[d] / m;
  t2[0] = n[1] * t1[2] - n[2] * t1[1];
  t2[1] = n[2] * t1[0] - n[0] * t1[2];
  t2[2] = n[0] * t1[1] - n[1] * t1[0];
}

// The closure's pair frame, fixed to the lattice.  D3Q19 and a sphere
// template centred on a lattice site are invariant under the 48 signed axis
// permutations of the cubic group, so a pair and its image under any of them
// have the same forces, mapped by the same operation (angular velocities and
// torques as pseudovectors).  P is the one (stable order by descending |n|,
// ties to the lower axis; sign + for n_k >= 0) that takes n into the
// fundamental domain nc = P n, nc_0 >= nc_1 >= nc_2 >= 0; the frame is
// pair_frame(nc) carried back by P^T: rows E[0] = n, E[1] = P^T t1(nc),
// E[2] = P^T t2(nc).  Returns det P (+-1): the pair-frame components are
// E dv for velocities and det P * E w for angular velocities, and forces
// and torques come back as E^T y and det P * E^T y.  Every pair of one
// lattice class (one separation vector up to the group) then has the same
// gap, nc and frame, and the same forces for the same pair-frame inputs.
__host__ __device__ inline double lattice_frame(const double n[3], double E[3][3], double nc[3]) {
  const double a[3] = {fabs(n[0]), fabs(n[1]), fabs(n[2])};
  int o[3] = {0, 1, 2};
  auto sw = [](int& x, int& y) { int t = x; x = y; y = t; };
  if (a[o[1]] > a[o[0]]) sw(o[0], o[1]);
  if (a[o[2]] > a[o[1]]) {
    sw(o[1], o[2]);
    if (a[o[1]] > a[o[0]]) sw(o[0], o[1]);
  }
  double sg[3];
  for (int k = 0; k < 3; ++k) sg[k] = n[k] >= 0.0 ? 1.0 : -1.0;
  for (int r = 0; r < 3; ++r) nc[r] = a[o[r]];
  double t1[3], t2[3];
  pair_frame(nc, t1, t2);
  for (int r = 0; r < 3; ++r) {
    E[0][o[r]] = n[o[r]];
    E[1][o[r]] = sg[o[r]] * t1[r];
    E[2][o[r]] = sg[o[r]] * t2[r];
  }
  // det P = parity of the permutation o times the product of the signs
  const int inv = (o[0] > o[1]) + (o[0] > o[2]) + (o[1] > o[2]);
  return ((inv & 1) ? -1.0 : 1.0) * sg[0] * sg[1] * sg[2];
}

}  // namespace lbx
