// lbx_closure.cu — learned lubrication / sub-resolution closure for sphere
// pairs (no counterpart in the reference; it attaches where the reference's
// analytic lubrication branch sits, addHertzian, kernels_fluid_PART.CUF:
// 1463-1501, which stays the fallback and the judge).
//
// Network: 13 -> 64 -> 64 -> 64 -> 12, SiLU, FP32.  Inputs, in the
// lattice-fixed pair frame E of spheres i < j (lattice_frame in
// lbx_closure.h: first axis n = (x_j - x_i)/|x_j - x_i|, transverse axes
// fixed by the cubic symmetry class of n, sign s = det of that class map):
//   gap/R, E (v_j - v_i), s E omega_i, s E omega_j, R, nc_1, nc_2
// (angular velocities in the lab frame; nc the sorted |n| components, which
// with the gap name the pair's lattice class).  Outputs: force and torque
// corrections on i and on j in the same frame (torques carry s).  Inputs and
// outputs are standardised with the mean / std stored after the weights.
// Training decays the Adam step size from lr to 0 as a half cosine over the
// optimiser steps of all epochs.
//
// Kernels
//   k_mlp_train  one thread-block cluster of 8 CTAs runs every epoch of
//                minibatch Adam on the whole data set: each CTA takes 8 of
//                the 64 samples of a minibatch (forward, backward, its
//                gradient in shared memory), the gradient is summed over the
//                cluster in rank order through distributed shared memory,
//                each CTA updates one slice of the parameters and writes it
//                into every CTA's copy.
//   k_mlp_infer  one warp per sample (pair), weights in shared memory.
//   k_pairs (lbx_particles.cu) / k_closure_pairs / k_closure_accum: per
//                step, the close pairs of each sphere (ascending index, listed
//                by the all-pairs force pass), the closure (or the
//                analytic lubrication when the pair leaves the training
//                envelope) and a fixed-order accumulation per sphere.
#include "lbx_device.cuh"
#include "lbx_closure.h"

#include <cooperative_groups.h>
#include <cmath>
#include <vector>

namespace lbx {

// ---------------------------------------------------------------------------
// training: a thread-block cluster of NCL CTAs, minibatch TB split over them
// ---------------------------------------------------------------------------
constexpr int TB = 64;              // minibatch
constexpr int TT = 256;             // threads per CTA
constexpr int NCL = 8;              // CTAs of the cluster (portable cluster size)
constexpr int TBC = TB / NCL;       // samples of a minibatch per CTA
constexpr int NP4 = (MlpLayout::NPARAM + 3) / 4 * 4;
constexpr int SLICE = (MlpLayout::NPARAM + NCL - 1) / NCL;  // parameters each CTA reduces and updates

struct TrainArgs {
  const float* X;   // n x DIN, standardised
  const float* T;   // n x DOUT, standardised
  int n;
  float* w;         // NPARAM (updated)
  float* loss;      // per epoch (may be null)
  float* grad_out;  // grad-only mode: NPARAM gradient of the first minibatch
  int epochs;
  float lr, beta1, beta2, eps;
  unsigned seed;
};

// Z[b][o] = sum_k A[b][k] W[o][k] + bias[o] for the CTA's TBC samples
__device__ void dense_fwd(const float* A, int K, const float* W, const float* bias, int O, float* Z) {
  for (int idx = threadIdx.x; idx < TBC * O; idx += TT) {
    const int b = idx / O, o = idx % O;
    const float* a = A + b * K;
    const float* wr = W + o * K;
    float s = bias[o];
    for (int k = 0; k < K; ++k) s = fmaf(a[k], wr[k], s);
    Z[idx] = s;
  }
}

// G[W][o][k] = sum_b dZ[b][o] A[b][k], G[bias][o] = sum_b dZ[b][o] (this CTA's samples, in order)
__device__ void dense_grad(const float* dZ, int O, const float* A, int K, float* GW, float* GB) {
  for (int idx = threadIdx.x; idx < O * K; idx += TT) {
    const int o = idx / K, k = idx % K;
    float s = 0.f;
#pragma unroll
    for (int b = 0; b < TBC; ++b) s = fmaf(dZ[b * O + o], A[b * K + k], s);
    GW[idx] = s;
  }
  for (int o = threadIdx.x; o < O; o += TT) {
    float s = 0.f;
#pragma unroll
    for (int b = 0; b < TBC; ++b) s += dZ[b * O + o];
    GB[o] = s;
  }
}

// dZp[b][k] = (sum_o dZ[b][o] W[o][k]) * silu'(Zp[b][k])
__device__ void dense_back(const float* dZ, int O, const float* W, const float* Zp, int K, float* dZp) {
  for (int idx = threadIdx.x; idx < TBC * K; idx += TT) {
    const int b = idx / K, k = idx % K;
    float s = 0.f;
    for (int o = 0; o < O; ++o) s = fmaf(dZ[b * O + o], W[o * K + k], s);
    dZp[idx] = s * dsilu(Zp[idx]);
  }
}

// Every epoch of minibatch Adam on the whole data set in one launch of one
// cluster.  Each CTA holds the weights, runs forward and backward for its
// TBC samples of the minibatch and keeps their gradient in its shared
// memory; after a cluster barrier CTA r sums slice r of the gradient over the
// CTAs in rank order (distributed shared memory reads), updates that slice
// with Adam (its moments stay in its shared memory) and writes the new
// values into every CTA's weights; a second barrier ends the step.  The
// minibatches, their order and the update are those of a single CTA running
// all TB samples; only the summation order of the gradient differs.
__global__ void __cluster_dims__(NCL, 1, 1) __launch_bounds__(TT) k_mlp_train(TrainArgs a) {
  namespace cg = cooperative_groups;
  using L = MlpLayout;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = int(cl.block_rank());
  extern __shared__ float sm[];
  float* W = sm;                       // NPARAM (replicated)
  float* G = W + NP4;                  // NPARAM: gradient of this CTA's samples
  float* Mo = G + NP4;                 // SLICE: Adam moments of this CTA's slice
  float* Vo = Mo + SLICE;
  float* X0 = Vo + SLICE;              // TBC x DIN
  float* Z1 = X0 + TBC * DIN;          // TBC x H pre-activations
  float* Z2 = Z1 + TBC * H;
  float* Z3 = Z2 + TBC * H;
  float* A1 = Z3 + TBC * H;            // TBC x H activations
  float* A2 = A1 + TBC * H;
  float* A3 = A2 + TBC * H;
  float* Y = A3 + TBC * H;             // TBC x DOUT
  float* D = Y + TBC * DOUT;           // TBC x DOUT: dL/dY
  float* E = D + TBC * DOUT;           // TBC x H: dL/dZ of the current layer
  float* F = E + TBC * H;              // TBC x H: dL/dZ of the layer below
  __shared__ float red[TT];
  __shared__ int idxs[TBC];
  __shared__ float part_loss;
  for (int i = threadIdx.x; i < L::NPARAM; i += TT) W[i] = a.w[i];
  for (int i = threadIdx.x; i < SLICE; i += TT) Mo[i] = Vo[i] = 0.f;
  const int lo = rank * SLICE, hi = min(L::NPARAM, lo + SLICE);
  __syncthreads();
  const int nb = (a.n + TB - 1) / TB;
  const bool grad_only = a.grad_out != nullptr;
  int t_adam = 0;
  for (int ep = 0; ep < (grad_only ? 1 : a.epochs); ++ep) {
    // epoch order: i -> (i * stride + off) mod n with stride coprime to n
    unsigned h = a.seed * 2654435761u + unsigned(ep) * 40503u + 12345u;
    int off = int(h % unsigned(a.n));
    int stride = 1 + int((h >> 8) % unsigned(a.n));
    while (true) {  // gcd(stride, n) == 1
      int x = stride, y = a.n;
      while (y) { int t = x % y; x = y; y = t; }
      if (x == 1) break;
      stride = stride % a.n + 1;
    }
    float ep_loss = 0.f;
    for (int bi = 0; bi < (grad_only ? 1 : nb); ++bi) {
      const int cnt = min(TB, a.n - bi * TB);
      for (int b = threadIdx.x; b < TBC; b += TT) {
        const int gb = rank * TBC + b;  // sample of the minibatch
        idxs[b] = grad_only ? min(gb, a.n - 1)
                            : int((long long)(bi * TB + min(gb, cnt - 1)) * stride % a.n + off) % a.n;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < TBC * DIN; i += TT) X0[i] = a.X[size_t(idxs[i / DIN]) * DIN + i % DIN];
      __syncthreads();
      // forward
      dense_fwd(X0, DIN, W + L::W0, W + L::B0, H, Z1);
      __syncthreads();
      for (int i = threadIdx.x; i < TBC * H; i += TT) A1[i] = silu(Z1[i]);
      __syncthreads();
      dense_fwd(A1, H, W + L::W1, W + L::B1, H, Z2);
      __syncthreads();
      for (int i = threadIdx.x; i < TBC * H; i += TT) A2[i] = silu(Z2[i]);
      __syncthreads();
      dense_fwd(A2, H, W + L::W2, W + L::B2, H, Z3);
      __syncthreads();
      for (int i = threadIdx.x; i < TBC * H; i += TT) A3[i] = silu(Z3[i]);
      __syncthreads();
      dense_fwd(A3, H, W + L::W3, W + L::B3, DOUT, Y);
      __syncthreads();
      // loss = mean over the minibatch's valid samples and outputs of (y - t)^2
      float part = 0.f;
      const float scale = 2.0f / float(cnt * DOUT);
      for (int i = threadIdx.x; i < TBC * DOUT; i += TT) {
        const int b = i / DOUT;
        const float d = (rank * TBC + b < cnt) ? Y[i] - a.T[size_t(idxs[b]) * DOUT + i % DOUT] : 0.f;
        part += d * d;
        D[i] = d * scale;
      }
      red[threadIdx.x] = part;
      __syncthreads();
      for (int st = TT / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
      }
      if (threadIdx.x == 0) part_loss = red[0];
      // backward: output layer, then the three hidden layers
      dense_grad(D, DOUT, A3, H, G + L::W3, G + L::B3);
      dense_back(D, DOUT, W + L::W3, Z3, H, E);
      __syncthreads();
      dense_grad(E, H, A2, H, G + L::W2, G + L::B2);
      dense_back(E, H, W + L::W2, Z2, H, F);
      __syncthreads();
      dense_grad(F, H, A1, H, G + L::W1, G + L::B1);
      dense_back(F, H, W + L::W1, Z1, H, E);
      __syncthreads();
      dense_grad(E, H, X0, DIN, G + L::W0, G + L::B0);
      cl.sync();  // every CTA's gradient and loss share are complete
      if (rank == 0 && threadIdx.x == 0)
        for (int r = 0; r < NCL; ++r) ep_loss += *cl.map_shared_rank(&part_loss, r);
      if (grad_only) {
        for (int i = lo + int(threadIdx.x); i < hi; i += TT) {
          float g = 0.f;
          for (int r = 0; r < NCL; ++r) g += cl.map_shared_rank(G, r)[i];
          a.grad_out[i] = g;
        }
        cl.sync();
        break;
      }
      // Adam on this CTA's slice; the new weights go to every CTA
      ++t_adam;
      const float c1 = 1.0f - powf(a.beta1, float(t_adam)), c2 = 1.0f - powf(a.beta2, float(t_adam));
      const float lr_t = 0.5f * a.lr * (1.0f + cospif(float(t_adam - 1) / float(a.epochs * nb)));
      for (int i = lo + int(threadIdx.x); i < hi; i += TT) {
        float gi = 0.f;
        for (int r = 0; r < NCL; ++r) gi += cl.map_shared_rank(G, r)[i];
        const float mi = a.beta1 * Mo[i - lo] + (1.0f - a.beta1) * gi;
        const float vi = a.beta2 * Vo[i - lo] + (1.0f - a.beta2) * gi * gi;
        Mo[i - lo] = mi;
        Vo[i - lo] = vi;
        const float wi = W[i] - lr_t * (mi / c1) / (sqrtf(vi / c2) + a.eps);
        for (int r = 0; r < NCL; ++r) cl.map_shared_rank(W, r)[i] = wi;
      }
      cl.sync();  // new weights everywhere; gradients free for the next step
    }
    if (rank == 0 && threadIdx.x == 0 && a.loss && !grad_only) a.loss[ep] = ep_loss / float(a.n * DOUT);
  }
  if (!grad_only && rank == 0)
    for (int i = threadIdx.x; i < L::NPARAM; i += TT) a.w[i] = W[i];
}

// ---------------------------------------------------------------------------
// inference: one warp per sample, weights (and normalisation) in shared memory
// ---------------------------------------------------------------------------
__global__ void k_mlp_infer(const float* __restrict__ Wg, const float* __restrict__ X, int n, float* Y) {
  extern __shared__ float sm[];
  float* W = sm;
  float* bufs = W + MlpLayout::TOTAL;
  load_infer_weights(Wg, W);
  __syncthreads();
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float* buf = bufs + warp * 2 * H;
  for (int s = blockIdx.x * nw + warp; s < n; s += gridDim.x * nw) {
    float x[DIN], y[DOUT];
    for (int k = 0; k < DIN; ++k) x[k] = X[size_t(s) * DIN + k];
    mlp_warp(W, x, y, buf);
    if ((threadIdx.x & 31) == 0)
      for (int o = 0; o < DOUT; ++o) Y[size_t(s) * DOUT + o] = y[o];
  }
}

// Launch of k_mlp_infer on device buffers (weights, n x DIN features, n x
// DOUT outputs) on the legacy default stream; used by entry points that
// manage their own device memory.
int closure_infer_launch(const float* dW, const float* dX, int n, float* dY) {
  using L = MlpLayout;
  const size_t smem = sizeof(float) * (size_t(L::TOTAL) + 8 * 2 * H);
  if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return LBX_ERR_CUDA;
  int blocks = (n + 7) / 8;
  if (blocks > 148 * 4) blocks = 148 * 4;
  k_mlp_infer<<<blocks, 256, smem>>>(dW, dX, n, dY);
  return cudaGetLastError() == cudaSuccess ? 0 : LBX_ERR_CUDA;
}

}  // namespace lbx

// ---------------------------------------------------------------------------
// host entry points (C ABI, include/lbx.h)
// ---------------------------------------------------------------------------
namespace {
struct Dev {
  void* p = nullptr;
  explicit Dev(size_t b) {
    if (b && cudaMalloc(&p, b) != cudaSuccess) p = nullptr;
  }
  ~Dev() {
    if (p) cudaFree(p);
  }
};
size_t train_smem() {
  return sizeof(float) * (2 * size_t(lbx::NP4) + 2 * size_t(lbx::SLICE) + lbx::TBC * lbx::DIN + 6 * lbx::TBC * lbx::H +
                          2 * lbx::TBC * lbx::DOUT + 2 * lbx::TBC * lbx::H);
}
int rc_of(cudaError_t e) { return e == cudaSuccess ? 0 : LBX_ERR_CUDA; }
}  // namespace

extern "C" {

int lbx_closure_init(float* weights, int32_t seed) {
  using L = lbx::MlpLayout;
  if (!weights) return LBX_ERR_ARG;
  // Glorot-uniform weights, zero biases, identity standardisation
  unsigned long long s = 0x9E3779B97F4A7C15ull ^ (unsigned long long)(seed);
  auto rnd = [&]() {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    return double(s >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int fan_out, int fan_in) {
    double lim = std::sqrt(6.0 / double(fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) weights[off + i] = float((2.0 * rnd() - 1.0) * lim);
  };
  for (int i = 0; i < L::TOTAL; ++i) weights[i] = 0.f;
  fill(L::W0, lbx::H, lbx::DIN);
  fill(L::W1, lbx::H, lbx::H);
  fill(L::W2, lbx::H, lbx::H);
  fill(L::W3, lbx::DOUT, lbx::H);
  for (int i = 0; i < lbx::DIN; ++i) weights[L::XSD + i] = 1.f;
  for (int i = 0; i < lbx::DOUT; ++i) weights[L::YSD + i] = 1.f;
  return 0;
}

int lbx_closure_train(float* weights, const float* X, const float* T, int32_t n, int32_t epochs, float lr,
                      int32_t seed, float* loss) {
  using L = lbx::MlpLayout;
  if (!weights || !X || !T || n < 1 || epochs < 1) return LBX_ERR_ARG;
  const size_t nx = size_t(n) * lbx::DIN, nt = size_t(n) * lbx::DOUT;
  Dev dX(nx * 4), dT(nt * 4), dW(size_t(L::TOTAL) * 4), dL(size_t(epochs) * 4);
  if (!dX.p || !dT.p || !dW.p || !dL.p) return LBX_ERR_ALLOC;
  // standardise with the statistics stored in the blob
  std::vector<float> Xs(nx), Ts(nt);
  for (size_t i = 0; i < nx; ++i) Xs[i] = (X[i] - weights[L::XMU + i % lbx::DIN]) / weights[L::XSD + i % lbx::DIN];
  for (size_t i = 0; i < nt; ++i) Ts[i] = (T[i] - weights[L::YMU + i % lbx::DOUT]) / weights[L::YSD + i % lbx::DOUT];
  int rc = rc_of(cudaMemcpy(dX.p, Xs.data(), nx * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dT.p, Ts.data(), nt * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dW.p, weights, size_t(L::TOTAL) * 4, cudaMemcpyHostToDevice));
  if (rc) return rc;
  lbx::TrainArgs a{(const float*)dX.p, (const float*)dT.p, n, (float*)dW.p, (float*)dL.p, nullptr, epochs, lr,
                   0.9f, 0.999f, 1e-8f, unsigned(seed)};
  size_t smem = train_smem();
  rc = rc_of(cudaFuncSetAttribute(lbx::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  if (rc) return rc;
  lbx::k_mlp_train<<<lbx::NCL, lbx::TT, smem>>>(a);  // one cluster
  rc = rc_of(cudaGetLastError());
  if (!rc) rc = rc_of(cudaDeviceSynchronize());
  if (!rc) rc = rc_of(cudaMemcpy(weights, dW.p, size_t(L::NPARAM) * 4, cudaMemcpyDeviceToHost));
  if (!rc && loss) rc = rc_of(cudaMemcpy(loss, dL.p, size_t(epochs) * 4, cudaMemcpyDeviceToHost));
  return rc;
}

int lbx_closure_grad(const float* weights, const float* Xs, const float* Ts, int32_t n, float* grad) {
  using L = lbx::MlpLayout;
  if (!weights || !Xs || !Ts || !grad || n < 1) return LBX_ERR_ARG;
  const size_t nx = size_t(n) * lbx::DIN, nt = size_t(n) * lbx::DOUT;
  Dev dX(nx * 4), dT(nt * 4), dW(size_t(L::TOTAL) * 4), dG(size_t(L::NPARAM) * 4);
  if (!dX.p || !dT.p || !dW.p || !dG.p) return LBX_ERR_ALLOC;
  int rc = rc_of(cudaMemcpy(dX.p, Xs, nx * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dT.p, Ts, nt * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dW.p, weights, size_t(L::TOTAL) * 4, cudaMemcpyHostToDevice));
  if (rc) return rc;
  lbx::TrainArgs a{(const float*)dX.p, (const float*)dT.p, n, (float*)dW.p, nullptr, (float*)dG.p, 1, 0.f,
                   0.9f, 0.999f, 1e-8f, 0u};
  size_t smem = train_smem();
  rc = rc_of(cudaFuncSetAttribute(lbx::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  if (rc) return rc;
  lbx::k_mlp_train<<<lbx::NCL, lbx::TT, smem>>>(a);  // one cluster
  rc = rc_of(cudaGetLastError());
  if (!rc) rc = rc_of(cudaDeviceSynchronize());
  if (!rc) rc = rc_of(cudaMemcpy(grad, dG.p, size_t(L::NPARAM) * 4, cudaMemcpyDeviceToHost));
  return rc;
}

int lbx_closure_infer(const float* weights, const float* X, int32_t n, float* Y) {
  using L = lbx::MlpLayout;
  if (!weights || !X || !Y || n < 1) return LBX_ERR_ARG;
  Dev dX(size_t(n) * lbx::DIN * 4), dY(size_t(n) * lbx::DOUT * 4), dW(size_t(L::TOTAL) * 4);
  if (!dX.p || !dY.p || !dW.p) return LBX_ERR_ALLOC;
  int rc = rc_of(cudaMemcpy(dX.p, X, size_t(n) * lbx::DIN * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dW.p, weights, size_t(L::TOTAL) * 4, cudaMemcpyHostToDevice));
  if (rc) return rc;
  size_t smem = sizeof(float) * (size_t(L::TOTAL) + 8 * 2 * lbx::H);
  rc = rc_of(cudaFuncSetAttribute(lbx::k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  if (rc) return rc;
  int blocks = (n + 7) / 8;
  if (blocks > 148 * 4) blocks = 148 * 4;
  lbx::k_mlp_infer<<<blocks, 256, smem>>>((const float*)dW.p, (const float*)dX.p, n, (float*)dY.p);
  rc = rc_of(cudaGetLastError());
  if (!rc) rc = rc_of(cudaDeviceSynchronize());
  if (!rc) rc = rc_of(cudaMemcpy(Y, dY.p, size_t(n) * lbx::DOUT * 4, cudaMemcpyDeviceToHost));
  return rc;
}

}  // extern "C"
