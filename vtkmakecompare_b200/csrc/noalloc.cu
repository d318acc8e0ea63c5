// noalloc.cu -- the spectral tridiagonal solve of SPN (mkp.f:223-260) for
// callers that cannot allocate GPU memory.
//
// Who needs this: a caller whose device memory is owned by someone else --
// a Fortran code whose arrays already live on the GPU (OpenACC / CUDA
// Fortran data regions hand us device pointers), a framework that reserves
// all device allocation to its own pool, or a time loop that must not hit
// cudaMalloc, which synchronises the whole device.  Such a caller passes
// device pointers for its inputs and outputs; the solve's scratch (the
// modified super-diagonal of every (kx,kz) system, tridiag.f:48) lives in a
// fixed array compiled into the library instead of being allocated.
//
// The array holds NSE_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB) on every GPU
// that loads the library, until the process exits.  It is shared by every
// call: a call writes each scratch value before reading it, so no clearing
// is needed, but two calls that overlap on the GPU (different streams or
// devices sharing a context) race on it and must be serialised by the caller.
//
// The array's device address is looked up once per device, on the first
// call with that device current, and cached for the life of the process.
// cudaDeviceReset destroys the context the address belongs to: a program
// that resets a device must not call this entry point on it afterwards.
#include <atomic>

#include "common.cuh"

namespace {

constexpr long kScratchDoubles = NSE_NOALLOC_SCRATCH_DOUBLES;
static __device__ __align__(256) double g_spn_scratch[kScratchDoubles];

// device address of g_spn_scratch per device, looked up on first use (host
// threads may race on the first lookup; they store the same address)
constexpr int kMaxDevices = 64;
static std::atomic<double*> g_scratch_ptr[kMaxDevices];

double* scratch_for_current_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  double* p = g_scratch_ptr[dev].load();
  if (!p) {
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_spn_scratch);
    if (e != cudaSuccess) {
      nse::set_error(NSE_ERR_CUDA, "nse_spn_noalloc: cudaGetSymbolAddress: %s",
                     cudaGetErrorString(e));
      return nullptr;
    }
    g_scratch_ptr[dev].store(p);
  }
  return p;
}

}  // namespace

extern "C" int nse_spn_noalloc(int nx, int ny, int nz, const double* AC, const double* KXZ,
                               double* PHIT, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !AC || !KXZ || !PHIT) {
    nse::set_error(NSE_ERR_ARG, "nse_spn_noalloc: bad arguments (nx=%d ny=%d nz=%d)", nx, ny, nz);
    return NSE_ERR_ARG;
  }
  const long H = nx / 2 + 1;
  if (H * (long)ny * (long)nz > kScratchDoubles) {
    nse::set_error(NSE_ERR_LIMIT,
                   "nse_spn_noalloc: (nx/2+1)*ny*nz = %ld exceeds the fixed scratch of %ld "
                   "values; use spn_ or the resident API for this size",
                   H * (long)ny * (long)nz, kScratchDoubles);
    return NSE_ERR_LIMIT;
  }
  if (nz > 65535) {  // nz is the launch grid's y dimension
    nse::set_error(NSE_ERR_LIMIT, "nse_spn_noalloc: nz = %d exceeds 65535", nz);
    return NSE_ERR_LIMIT;
  }
  if (!nse::ensure_device()) return NSE_ERR_CUDA;
  // an error left by the caller's earlier asynchronous work is reported as
  // such and left in place (cudaPeekAtLastError does not clear it)
  cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    nse::set_error(NSE_ERR_CUDA, "nse_spn_noalloc: a CUDA error is pending from earlier work: %s",
                   cudaGetErrorString(pending));
    return NSE_ERR_CUDA;
  }
  double* sc = scratch_for_current_device();
  if (!sc) {
    if (nse_last_status() == NSE_OK)
      nse::set_error(NSE_ERR_CUDA, "nse_spn_noalloc: no scratch on this device");
    return NSE_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  // PHIT(0:nx/2, 0:ny+1, 0:nz+1) complex: plane J = 1 starts H values in
  nse::launch_spn_view((int)H, ny, nz, PHIT + 2 * H, H, H * (ny + 2), sc, H, H * (long)ny, AC,
                       KXZ, true, false, s);
  cudaError_t e = cudaGetLastError();  // nothing was pending: this is the launch's
  if (e != cudaSuccess) {
    nse::set_error(NSE_ERR_CUDA, "nse_spn_noalloc: launch: %s", cudaGetErrorString(e));
    return NSE_ERR_CUDA;
  }
  return NSE_OK;
}
