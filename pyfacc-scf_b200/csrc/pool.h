// Process-wide pools of device memory, GPU contexts and basis files (pool.cpp).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <memory>
#include <string>
#include <vector>

namespace pyfacc {

// Device memory: blocks come back from pool_free to a per-device free list
// (at most 8 GiB cached per device) and are reused by later requests.
void* pool_alloc(size_t bytes, size_t* got);
void pool_free(void* p, size_t bytes);
void pool_trim(int device);

// One stream with its cuBLAS and cuSOLVER handles and two timing events.
struct GpuContext {
  int device = 0;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // a second stream for work that may overlap the main stream's (the FP32
  // half of a mixed Fock build or gradient), forked and joined by events
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // pinned host words for the per-iteration readbacks (asynchronous copies,
  // so work queued after them runs while the host waits on `ready`)
  double* pinned = nullptr;
  cudaEvent_t ready = nullptr;
};
constexpr int PINNED_DOUBLES = 256;
// layout of GpuContext::pinned: [0, 72) energy, errors and DIIS overlaps of
// an SCF iteration; [128, 136) the purification outcome; [200, 202) the
// overlap factor's smallest pivot and status
constexpr int PURIFY_PINNED = 128;
constexpr int ORTHO_PINNED = 200;
GpuContext context_acquire(int device);   // the current device must be `device`
void context_release(const GpuContext& c);

// Lines of a basis-set file, read once per process.
std::shared_ptr<const std::vector<std::string>> basis_lines(const std::string& path,
                                                            std::vector<std::string> (*reader)(const std::string&));

}  // namespace pyfacc
