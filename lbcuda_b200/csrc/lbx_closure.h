// lbx_closure.h — the learned pair closure shared by its training/inference
// kernels (lbx_closure.cu) and the particle step (lbx_particles.cu):
// network dimensions, the weight-blob layout, the warp-level forward pass and
// the pair frame.
#pragma once
#include <cuda_runtime.h>

#include "../../include/lbx.h"

namespace lbx {
constexpr int DIN = 11, H = 64, DOUT = 12;

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

}  // namespace lbx
