// The engine of libcfd2lcs_b200 (class Engine in engine_impl.cuh): this file instantiates it
// with the velocity stored in the interface type (plain form) and holds the scratch table of the
// allocation-free entry point; engine_mixed.cu instantiates the mixed-precision form (FP32
// velocity) of the double library, so that the two compile in parallel.
#include "engine_impl.cuh"

namespace cfd2lcs {

// ---------------------------------------------------------------------------------------
// Scratch of the allocation-free reconstruction entry point: the table of sub-flow-map
// pointers the composition kernel reads, as a file-scope device array instead of an
// allocated buffer.  Every GPU that loads the library holds these 6 KiB until exit; all
// calls share the table (calls that overlap on the GPU race on it).
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) const void *g_noalloc_submap_table[3 * NOALLOC_MAX_SUBMAPS];

// Device address of the table on device dev, looked up once per device with that device
// current (host code must not pass the symbol itself to a kernel: on the host it is only a
// stand-in).  The cache is filled under a lock, so first calls from several host threads do
// not race on it; the caller's current device is restored afterwards.
bool noalloc_table_address(int dev, void **out, std::string &msg) {
  static std::mutex lock;
  static void *addr[64] = {nullptr};
  if (dev < 0 || dev >= 64) {
    msg = "reconstruct_noalloc: device index out of range";
    return false;
  }
  std::lock_guard<std::mutex> guard(lock);
  if (!addr[dev]) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess && cur != dev) e = cudaSetDevice(dev);
    void *p = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_noalloc_submap_table);
    if (cur >= 0 && cur != dev) cudaSetDevice(cur);
    if (e != cudaSuccess || !p) {
      msg = std::string("reconstruct_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return false;
    }
    addr[dev] = p;
  }
  *out = addr[dev];
  return true;
}

#ifndef CFD2LCS_SP
std::unique_ptr<EngineBase> make_engine_mixed(const Options *opt);  // engine_mixed.cu
#endif

std::unique_ptr<EngineBase> make_engine(const Options *opt) {
#ifndef CFD2LCS_SP
  if (opt->mixed_precision) return make_engine_mixed(opt);
#else
  if (opt->mixed_precision) return std::unique_ptr<EngineBase>(new Engine<float>(opt));
#endif
  return std::unique_ptr<EngineBase>(new Engine<lcsdata_t>(opt));
}

}  // namespace cfd2lcs
