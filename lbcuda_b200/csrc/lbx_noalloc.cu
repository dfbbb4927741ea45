// lbx_noalloc.cu — closure inference without any device allocation (no
// counterpart in the reference).
//
// lbx_closure_infer allocates and frees its device buffers on every call.  A
// caller that must not allocate inside its run loop (device memory reserved
// up front for the lattice, with nothing left for a late cudaMalloc to find;
// a fixed device footprint required for the whole run) cannot use it.  This
// variant stages weights, features and outputs in one file-scope device
// array of fixed size and runs the same inference kernel.
//
//   capacity:  LBX_CLOSURE_NOALLOC_MAX pairs (4096); larger n is rejected
//              with LBX_ERR_ARG before any device work
//   scratch:   weights (LBX_CLOSURE_NWEIGHTS floats, padded to 10048), then
//              X (MAX x 13), then Y (MAX x 12): 449,792 bytes per device
//   zeroing:   none needed; every call overwrites the weights and the n
//              feature rows it uses, and the kernel writes every output row
//              that is copied back
//   setup:     the first call on a device, with that device current, looks
//              up the array's address (cudaGetSymbolAddress) and keeps it.
//              With lazy module loading (the CUDA default) that lookup is
//              also where the library's module, and with it this array, gets
//              its device memory, so make the first call on each device
//              before reserving device memory up front and before any stream
//              capture
//   lifetime:  the kept address belongs to the device's primary context;
//              after cudaDeviceReset the entry point is not valid any more in
//              this process (the address would be stale)
//   races:     calls share the array of their device; calls that overlap in
//              time on one device (several host threads) race, so such
//              callers serialise them
#include <mutex>

#include "lbx_device.cuh"

namespace lbx {
int closure_infer_launch(const float* dW, const float* dX, int n, float* dY);
}

namespace {

constexpr int kWPad = 10048;  // LBX_CLOSURE_NWEIGHTS rounded up to 256 bytes
constexpr int kDin = 13, kDout = 12;
constexpr size_t kScratchFloats = size_t(kWPad) + size_t(LBX_CLOSURE_NOALLOC_MAX) * (kDin + kDout);
static_assert(LBX_CLOSURE_NWEIGHTS <= kWPad, "weight blob exceeds its scratch slot");

__device__ __align__(256) float g_infer_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

// address of this device's scratch (looked up once per device)
int scratch_of_current_device(float** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return LBX_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return LBX_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_infer_scratch) != cudaSuccess || !p) return LBX_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

int rc_of(cudaError_t e) { return e == cudaSuccess ? 0 : LBX_ERR_CUDA; }

}  // namespace

extern "C" {

int lbx_closure_infer_noalloc(const float* weights, const float* X, int32_t n, float* Y) {
  if (!weights || !X || !Y || n < 1 || n > LBX_CLOSURE_NOALLOC_MAX) return LBX_ERR_ARG;
  float* base = nullptr;
  int rc = scratch_of_current_device(&base);
  if (rc) return rc;
  float* dW = base;
  float* dX = base + kWPad;
  float* dY = dX + size_t(LBX_CLOSURE_NOALLOC_MAX) * kDin;
  // The copies and the launch all go to the legacy default stream, so the
  // blocking copy of Y back waits for the kernel without a separate
  // synchronise; a move of the launch to another stream needs one.
  rc = rc_of(cudaMemcpy(dW, weights, size_t(LBX_CLOSURE_NWEIGHTS) * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = rc_of(cudaMemcpy(dX, X, size_t(n) * kDin * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = lbx::closure_infer_launch(dW, dX, n, dY);
  if (!rc) rc = rc_of(cudaMemcpy(Y, dY, size_t(n) * kDout * 4, cudaMemcpyDeviceToHost));
  return rc;
}

}  // extern "C"
