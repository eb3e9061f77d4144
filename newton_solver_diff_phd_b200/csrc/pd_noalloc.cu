// Allocation-free application of the inverse factor: out = S^T (S rhs).
//
// Some callers cannot call cudaMalloc at the moment they need a solve: code
// running while a stream is being captured into a CUDA graph, engines and
// plugins whose host owns every device allocation through its own pool, and
// real-time loops that must not take the driver's allocation lock. For them
// pd_apply_inverse_static computes the same product as pd_apply_inverse, but
// keeps its one intermediate vector y = S rhs in a file-scope device array
// instead of solver-owned scratch. The caller passes rhs and out; the factor
// is the one the solver uploaded in pd_build.
//
// The array holds at most kStaticScratchParticles particles (3 doubles each,
// 1.5 MiB) and stays resident on every GPU that loads the library until the
// process exits. All calls share it, so calls whose kernels overlap on the
// GPU (different streams, or different solvers on one device without
// ordering) race on it; serialise them. The array keeps the previous call's
// contents; every entry this call reads is written first by this call.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/pd_b200.h"
#include "pd_device.cuh"

namespace {

constexpr int kStaticScratchParticles = 65536;
constexpr int kMaxDevices = 64;

// One vec3 of float64 per particle: the intermediate y = S rhs.
static __device__ __align__(256) double g_static_scratch[3 * kStaticScratchParticles];

// Device address of g_static_scratch, looked up once per device.
void* g_scratch_address[kMaxDevices] = {};
std::mutex g_scratch_mutex;

__global__ void static_spmv_kernel(const int* __restrict__ off, const int* __restrict__ col,
                                   const double* __restrict__ val, const double* __restrict__ vec, double* out,
                                   int rows) {
  const int lane = threadIdx.x & 31;
  const int warps_total = (gridDim.x * blockDim.x) >> 5;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps_total) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int k = off[row] + lane; k < off[row + 1]; k += 32) {
      const double value = val[k];
      const int c = col[k];
      sx += value * vec[3 * c];
      sy += value * vec[3 * c + 1];
      sz += value * vec[3 * c + 2];
    }
    sx = pdb200::warp_sum(sx);
    sy = pdb200::warp_sum(sy);
    sz = pdb200::warp_sum(sz);
    if (lane == 0) {
      out[3 * row] = sx;
      out[3 * row + 1] = sy;
      out[3 * row + 2] = sz;
    }
  }
}

}  // namespace

// Defined in pd_solver.cu: the factor arrays of a built solver (device
// pointers) and the particle count of any solver.
int pd_internal_factor(PdSolver* solver, int* device, int* rows, const int** s_off, const int** s_col,
                       const double** s_val, const int** st_off, const int** st_col, const double** st_val);
int pd_internal_particles(const PdSolver* solver);
int pd_internal_fail(int code, const char* message);

namespace {

// Makes the solver's device current for the call and puts the caller's
// device back on every return path: callers that own their allocator also
// own the current-device setting of their thread.
class DeviceScope {
 public:
  cudaError_t enter(int device) {
    cudaError_t status = cudaGetDevice(&previous_);
    if (status != cudaSuccess) return status;
    entered_ = true;
    return previous_ == device ? cudaSuccess : cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (entered_) cudaSetDevice(previous_);
  }

 private:
  int previous_ = 0;
  bool entered_ = false;
};

}  // namespace

// Device address of the scratch array on `device` (the current device),
// resolved on the first request and cached.
cudaError_t static_scratch_address(int device, void** address) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_address[device] == nullptr) {
    const cudaError_t status = cudaGetSymbolAddress(&g_scratch_address[device], g_static_scratch);
    if (status != cudaSuccess) {
      g_scratch_address[device] = nullptr;
      return status;
    }
  }
  *address = g_scratch_address[device];
  return cudaSuccess;
}

// Called by pd_build (never inside stream capture) so that a first
// pd_apply_inverse_static inside a capture finds the address resolved.
int pd_internal_resolve_static_scratch(int device) {
  if (device < 0 || device >= kMaxDevices) return pd_internal_fail(PD_ERR_INVALID, "device ordinal out of range");
  void* address = nullptr;
  const cudaError_t status = static_scratch_address(device, &address);
  if (status != cudaSuccess)
    return pd_internal_fail(PD_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(status)).c_str());
  return PD_OK;
}

extern "C" int pd_apply_inverse_static(PdSolver* solver, const double* rhs, double* out, void* stream) {
  if (solver == nullptr || rhs == nullptr || out == nullptr) return pd_internal_fail(PD_ERR_INVALID, "null argument");
  // The size limit is checked first, so that an oversized solver is refused
  // whether or not its factor has been built.
  const int particles = pd_internal_particles(solver);
  if (particles > kStaticScratchParticles) {
    return pd_internal_fail(PD_ERR_INVALID,
                            ("pd_apply_inverse_static handles at most " + std::to_string(kStaticScratchParticles) +
                             " particles; this solver has " + std::to_string(particles))
                                .c_str());
  }
  int device = 0, rows = 0;
  const int *s_off = nullptr, *s_col = nullptr, *st_off = nullptr, *st_col = nullptr;
  const double *s_val = nullptr, *st_val = nullptr;
  if (int status = pd_internal_factor(solver, &device, &rows, &s_off, &s_col, &s_val, &st_off, &st_col, &st_val)) {
    return status;
  }
  if (rows == 0) return PD_OK;  // nothing to apply; a zero-block launch would be an error
  if (device < 0 || device >= kMaxDevices) return pd_internal_fail(PD_ERR_INVALID, "device ordinal out of range");
  DeviceScope scope;
  cudaError_t status = scope.enter(device);
  if (status != cudaSuccess) return pd_internal_fail(PD_ERR_CUDA, cudaGetErrorString(status));
  void* scratch = nullptr;
  status = static_scratch_address(device, &scratch);  // resolved by pd_build already
  if (status != cudaSuccess)
    return pd_internal_fail(PD_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(status)).c_str());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = (rows * 32 + pdb200::kBlock - 1) / pdb200::kBlock;
  double* y = static_cast<double*>(scratch);
  static_spmv_kernel<<<blocks, pdb200::kBlock, 0, st>>>(s_off, s_col, s_val, rhs, y, rows);
  static_spmv_kernel<<<blocks, pdb200::kBlock, 0, st>>>(st_off, st_col, st_val, y, out, rows);
  status = cudaGetLastError();
  if (status != cudaSuccess) return pd_internal_fail(PD_ERR_CUDA, cudaGetErrorString(status));
  return PD_OK;
}
