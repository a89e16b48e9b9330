// tsn_fft_adjoint_image_static: the adjoint FFT endpoint without any device allocation.
//
// Some callers cannot call cudaMalloc: real-time or embedded hosts whose device allocator
// is frozen after start-up, services that reserve all device memory up front, and plug-ins
// that run inside a host application which owns the device memory pool.  They cannot
// create a plan (a plan allocates its packs and workspaces), so this entry point takes
// every input and output from the caller and keeps its only intermediate -- the
// inverse-FFT half-transformed grid, G*N*C complex values -- in a file-scope device array
// of fixed size.
//
// Limits and behaviour:
//   * grid_size * im_size * coils <= kStaticScratchElems (1 Mi complex = 8 MiB), which
//     covers 512 x 256 x 8; larger shapes return TSN_ERR_SHAPE.
//   * The scratch array is shared by every call in the process on a given device and keeps
//     the last call's contents.  Each call overwrites all of the scratch it reads, so
//     nothing has to start at zero; calls that overlap on the GPU (different streams, no
//     ordering) race on it and must be serialized by the caller.
//   * The first call on a device does the set-up for the device that is current at that
//     call: it looks up the device addresses of the arrays with cudaGetSymbolAddress and
//     fills the twiddle tables of every supported grid size (128, 256, 384, 512, 640 and
//     1024 points, one table each).  Make that first call before any stream capture
//     begins.  Later calls only read the tables, so calls of different grid sizes in
//     stream order need no further ordering.
//   * Every GPU that loads the library holds the arrays until the process exits.
#include <cmath>
#include <cstdint>
#include <initializer_list>
#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"

namespace {

constexpr int64_t kStaticScratchElems = int64_t(1) << 20;  // complex elements
constexpr int kMaxGrid = 1024;
constexpr int kMaxDevices = 64;
// Supported grid sizes and the offset of each one's table in g_static_twiddle.
constexpr int kGridSizes[] = {128, 256, 384, 512, 640, 1024};
constexpr int kNumGrids = sizeof(kGridSizes) / sizeof(kGridSizes[0]);
constexpr int kTwiddleElems = 128 + 256 + 384 + 512 + 640 + 1024;

static __device__ __align__(256) float2 g_static_scratch[kStaticScratchElems];
static __device__ __align__(256) float2 g_static_twiddle[kTwiddleElems];
static __device__ __align__(256) tsn::CgState g_static_state;

int twiddle_offset(int grid_size) {
  int off = 0;
  for (int i = 0; i < kNumGrids; ++i) {
    if (kGridSizes[i] == grid_size) return off;
    off += kGridSizes[i];
  }
  return -1;
}

struct DeviceSetup {
  float2* scratch = nullptr;
  float2* twiddle = nullptr;  // all grid sizes' tables, kGridSizes order
  tsn::CgState* state = nullptr;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

[[noreturn]] void cuda_fail(cudaError_t e, const char* what) {
  tsn::fail(TSN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceSetup& setup_device(int device, cudaStream_t s) {
  if (device < 0 || device >= kMaxDevices) tsn::fail(TSN_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& d = g_setup[device];
  cudaError_t e;
  if (!d.scratch) {  // d.scratch is set last: a set-up that failed part way is redone
    void* p = nullptr;
    void* p_scratch = nullptr;
    if ((e = cudaGetSymbolAddress(&p_scratch, g_static_scratch)) != cudaSuccess)
      cuda_fail(e, "cudaGetSymbolAddress(scratch)");
    if ((e = cudaGetSymbolAddress(&p, g_static_twiddle)) != cudaSuccess) cuda_fail(e, "cudaGetSymbolAddress(twiddle)");
    d.twiddle = static_cast<float2*>(p);
    if ((e = cudaGetSymbolAddress(&p, g_static_state)) != cudaSuccess) cuda_fail(e, "cudaGetSymbolAddress(state)");
    d.state = static_cast<tsn::CgState*>(p);
    tsn::CgState init{};
    init.sigma_y = 1.0f;  // unit sample scale for the plain adjoint epilogue
    if ((e = cudaMemcpyToSymbol(g_static_state, &init, sizeof init)) != cudaSuccess) cuda_fail(e, "state init");
    // exp(-2 pi i k / G) for every supported G, written once: no call after this one
    // writes the tables
    std::vector<float2> tw;
    tw.reserve(kTwiddleElems);
    for (int i = 0; i < kNumGrids; ++i) {
      const int g = kGridSizes[i];
      for (int k = 0; k < g; ++k) {
        const double a = -2.0 * M_PI * k / g;
        tw.push_back(make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a))));
      }
    }
    if ((e = cudaMemcpyToSymbol(g_static_twiddle, tw.data(), sizeof(float2) * tw.size())) != cudaSuccess)
      cuda_fail(e, "twiddle init");
    tsn::set_twiddle_constants(s);
    d.scratch = static_cast<float2*>(p_scratch);
  }
  return d;
}

}  // namespace

namespace tsn {
tsn_status guard_status(const std::exception& e);
}

extern "C" tsn_status tsn_fft_adjoint_image_static(int32_t im_size, int32_t grid_size, int32_t coils, int32_t centered,
                                                   const void* grid_c64, const void* smaps, const float* scaling,
                                                   void* x, tsn_stream_t stream) {
  try {
    if (!grid_c64 || !scaling || !x) tsn::fail(TSN_ERR_ARG, "NULL argument");
    if (!tsn::fft_grid_supported(grid_size) || grid_size > kMaxGrid || twiddle_offset(grid_size) < 0)
      tsn::fail(TSN_ERR_UNSUPPORTED, "grid size must be 128, 256, 384, 512, 640 or 1024");
    if (im_size <= 0 || im_size % 4 || im_size > grid_size)
      tsn::fail(TSN_ERR_SHAPE, "need an image size that is a multiple of 4 and <= grid size");
    for (const void* p : {grid_c64, static_cast<const void*>(scaling), smaps, static_cast<const void*>(x)})
      if (reinterpret_cast<uintptr_t>(p) & 15u) tsn::fail(TSN_ERR_ARG, "device arrays must be 16-byte aligned");
    if (coils < 4 || coils > 16 || coils % 4) tsn::fail(TSN_ERR_UNSUPPORTED, "coil count must be 4, 8, 12 or 16");
    const int64_t need = static_cast<int64_t>(grid_size) * im_size * coils;
    if (need > kStaticScratchElems)
      tsn::fail(TSN_ERR_SHAPE, "grid_size * im_size * coils = " + std::to_string(need) +
                                   " exceeds the static scratch of " + std::to_string(kStaticScratchElems) +
                                   " complex elements");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) cuda_fail(e, "cudaGetDevice");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    DeviceSetup& d = setup_device(device, s);
    tsn::FftArgs f;
    f.N = im_size;
    f.G = grid_size;
    f.C = coils;
    f.shift = centered ? im_size / 2 : 0;
    f.tw = d.twiddle + twiddle_offset(grid_size);
    f.scaling = scaling;
    f.smaps = static_cast<const float2*>(smaps);
    tsn::launch_inv_cols(f, static_cast<const float2*>(grid_c64), d.scratch, s);
    tsn::launch_inv_rows(f, d.scratch, static_cast<float2*>(x), 0, nullptr, nullptr, nullptr, nullptr, d.state, 0,
                         1.0f, 0.f, s);
    if ((e = cudaGetLastError()) != cudaSuccess) cuda_fail(e, "launch");
    return TSN_OK;
  } catch (const std::exception& ex) {
    return tsn::guard_status(ex);
  }
}
