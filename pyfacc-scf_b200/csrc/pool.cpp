// Process-wide reuse of the expensive per-call resources, so that a call
// through the C ABI (pyfacc_run, run_scf_c) costs little more than its GPU
// work: device memory blocks (a size-ordered free list per device), the
// stream + cuBLAS + cuSOLVER triple of a system (a free list per device) and
// parsed basis-set files.  Everything is guarded by one mutex; blocks and
// handles return to the pools when a system is destroyed.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <map>
#include <mutex>
#include <vector>

#include "engine.h"
#include "pool.h"

namespace pyfacc {

namespace {
std::mutex g_pool_mu;
// device -> (bytes -> blocks)
std::map<int, std::multimap<size_t, void*>> g_free_blocks;
std::map<int, std::vector<GpuContext>> g_free_ctx;
std::map<std::string, std::shared_ptr<const std::vector<std::string>>> g_basis_text;
constexpr size_t kMaxCachedBytesPerDevice = size_t(8) << 30;
std::map<int, size_t> g_cached_bytes;
}  // namespace

void* pool_alloc(size_t bytes, size_t* got) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto& fl = g_free_blocks[dev];
    auto it = fl.lower_bound(bytes);
    // reuse a block that is not more than twice the request
    if (it != fl.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
      void* p = it->second;
      *got = it->first;
      g_cached_bytes[dev] -= it->first;
      fl.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    // give the cached blocks of this device back and retry once
    (void)cudaGetLastError();
    pool_trim(dev);
    PF_CUDA(cudaMalloc(&p, bytes));
  }
  *got = bytes;
  return p;
}

void pool_free(void* p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  if (cudaPointerAttributes a; cudaPointerGetAttributes(&a, p) == cudaSuccess) dev = a.device;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_cached_bytes[dev] + bytes > kMaxCachedBytesPerDevice) {
    cudaFree(p);
    return;
  }
  g_free_blocks[dev].emplace(bytes, p);
  g_cached_bytes[dev] += bytes;
}

void pool_trim(int dev) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (auto& kv : g_free_blocks[dev]) cudaFree(kv.second);
  g_free_blocks[dev].clear();
  g_cached_bytes[dev] = 0;
}

GpuContext context_acquire(int dev) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto& v = g_free_ctx[dev];
    if (!v.empty()) {
      GpuContext c = v.back();
      v.pop_back();
      return c;
    }
  }
  GpuContext c;
  c.device = dev;
  PF_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  if (cublasCreate(&c.cublas) != CUBLAS_STATUS_SUCCESS) throw Error(PYFACC_ERR_CUDA, "cublasCreate failed");
  if (cublasSetStream(c.cublas, c.stream) != CUBLAS_STATUS_SUCCESS) throw Error(PYFACC_ERR_CUDA, "cublasSetStream failed");
  if (cusolverDnCreate(&c.cusolver) != CUSOLVER_STATUS_SUCCESS) throw Error(PYFACC_ERR_CUDA, "cusolverDnCreate failed");
  if (cusolverDnSetStream(c.cusolver, c.stream) != CUSOLVER_STATUS_SUCCESS)
    throw Error(PYFACC_ERR_CUDA, "cusolverDnSetStream failed");
  PF_CUDA(cudaEventCreate(&c.ev0));
  PF_CUDA(cudaEventCreate(&c.ev1));
  PF_CUDA(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
  PF_CUDA(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
  PF_CUDA(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
  PF_CUDA(cudaEventCreateWithFlags(&c.ready, cudaEventDisableTiming));
  PF_CUDA(cudaMallocHost(&c.pinned, PINNED_DOUBLES * sizeof(double)));
  return c;
}

void context_release(const GpuContext& c) {
  if (!c.stream) return;
  cudaStreamSynchronize(c.stream);
  if (c.side) cudaStreamSynchronize(c.side);
  std::lock_guard<std::mutex> lk(g_pool_mu);
  g_free_ctx[c.device].push_back(c);
}

std::shared_ptr<const std::vector<std::string>> basis_lines(const std::string& path,
                                                            std::vector<std::string> (*reader)(const std::string&)) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_basis_text.find(path);
    if (it != g_basis_text.end()) return it->second;
  }
  auto v = std::make_shared<const std::vector<std::string>>(reader(path));
  std::lock_guard<std::mutex> lk(g_pool_mu);
  g_basis_text[path] = v;
  return v;
}

}  // namespace pyfacc
