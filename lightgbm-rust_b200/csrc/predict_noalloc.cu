// Batched raw-score prediction from host buffers that allocates no device
// memory: lgbm_b200_predict_noalloc.
//
// lgbm_b200_predict with host buffers allocates device staging for the
// feature rows and the scores (on its first call, and again whenever a
// larger batch arrives). Some callers cannot
// allocate at prediction time: a serving process that gives all device memory
// it does not hold to another allocator up front (a framework's caching
// allocator, a fixed memory budget) gets out-of-memory there, and a
// latency-bound serving thread must not wait on the allocator's locks or on
// the device-wide synchronisation that freeing memory can bring. This entry
// point instead stages the rows and the scores through one fixed array in
// device global memory, compiled into the library, in chunks of rows.
//
// The array is shared by every call on a device. Calls that overlap in time
// on the same device (from several host threads, or with several forests)
// race on it and give wrong scores: serialise them. Nothing in the array has
// to start at zero: each chunk's rows are copied in before the kernel reads
// them and every score is written before it is copied out.
//
// The first call on a device, with that device current, resolves the array's
// device address with cudaGetSymbolAddress (which also loads the library's
// device code on that device); make that first call before capturing any
// stream on the device. The calling thread's current device is the same
// before and after a call.
#include <mutex>

#include "learner_impl.h"

namespace lgbm_b200 {

// 16 MiB: 139,808 rows of 28 features per chunk for one class.
constexpr size_t kPredictStageBytes = size_t(16) << 20;
constexpr int kMaxStageDevices = 64;

static __device__ __align__(256) unsigned char g_predict_stage[kPredictStageBytes];

static unsigned char* g_stage_ptr[kMaxStageDevices];
static cudaError_t g_stage_err[kMaxStageDevices];
static std::once_flag g_stage_once[kMaxStageDevices];

// Device address of the staging array on `device`, resolved once per device
// with that device current.
static Status stage_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxStageDevices)
    return Status(LGBM_B200_ERR_INVALID_PARAMETER, "predict_noalloc: device ordinal above 63");
  std::call_once(g_stage_once[device], [device] {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_predict_stage);
    g_stage_err[device] = e;
    g_stage_ptr[device] = e == cudaSuccess ? static_cast<unsigned char*>(p) : nullptr;
  });
  if (g_stage_err[device] != cudaSuccess)
    return Status(LGBM_B200_ERR_CUDA,
                  std::string("predict_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(g_stage_err[device]));
  *out = g_stage_ptr[device];
  return Status();
}

}  // namespace lgbm_b200

using namespace lgbm_b200;

extern "C" {

namespace {

// Restores the calling thread's current device when the call returns, so a
// serving thread that works on another device keeps it.
struct DeviceRestore {
  int prev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

int lgbm_b200_predict_noalloc(LgbmB200Forest* F, const float* X, int64_t nrow, int32_t ncol, double* out) {
  if (!F || !X || !out || nrow < 0 || ncol <= 0)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER, "predict_noalloc: bad argument"));
  int device;
  cudaStream_t s;
  const DForest* f;
  int32_t ntpi;
  forest_parts(F, &device, &s, &f, &ntpi);
  // a chunk is [rows x ncol] f32 rows, then [rows x ntpi] f64 scores at the next 256-byte boundary
  const size_t row_bytes = sizeof(float) * (size_t)ncol + sizeof(double) * (size_t)ntpi;
  const size_t usable = kPredictStageBytes - 256;
  if (row_bytes > usable)
    return fail(Status(LGBM_B200_ERR_INVALID_PARAMETER,
                       "predict_noalloc: one row needs " + std::to_string(row_bytes) +
                           " staging bytes (4 x ncol + 8 x num_tree_per_iteration); the static staging array "
                           "holds 16 MiB"));
  if (nrow == 0) return LGBM_B200_OK;
  DeviceRestore restore;
  if (cudaSetDevice(device) != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, "cudaSetDevice"));
  unsigned char* stage;
  Status st = stage_address(device, &stage);
  if (!st.ok()) return fail(st);
  const int64_t chunk = (int64_t)(usable / row_bytes);
  float* xs = reinterpret_cast<float*>(stage);
  cudaError_t e = cudaSuccess;
  for (int64_t r0 = 0; r0 < nrow && e == cudaSuccess; r0 += chunk) {
    const int64_t m = std::min(chunk, nrow - r0);
    const size_t x_bytes = sizeof(float) * (size_t)m * (size_t)ncol;
    double* os = reinterpret_cast<double*>(stage + ((x_bytes + 255) / 256) * 256);
    // all three steps run in order on the forest's stream, so the next chunk's
    // rows overwrite the array only after this chunk's kernel and copy-out
    e = cudaMemcpyAsync(xs, X + r0 * ncol, x_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_predict(*f, xs, m, ncol, os, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out + r0 * ntpi, os, sizeof(double) * (size_t)m * ntpi, cudaMemcpyDeviceToHost, s);
  }
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return fail(Status(LGBM_B200_ERR_CUDA, cudaGetErrorString(e)));
  return LGBM_B200_OK;
}

}  // extern "C"
