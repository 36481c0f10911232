// cib_rve_pcg_noalloc: the periodic-RVE PCG solve for callers that must not allocate
// device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a memory pool's or a caching
// allocator's own hooks (where allocating would re-enter the allocator), host frameworks
// that forbid device allocations once they have partitioned device memory up front, and
// hot loops with a strict no-allocation budget.  cib_rve_pcg needs three work vectors
// (r, p, Ap) besides its inputs and outputs; this variant keeps them in one array that is
// compiled into the library, so the call itself allocates nothing.
//
// The array has a fixed size (3 x CIB_PCG_NOALLOC_MAX_VEC doubles = 1.5 MiB) and exists
// once on every GPU that loads the library, until the process exits.  All calls on a
// device share it and it keeps whatever the last call left there; the solver overwrites
// every entry it reads before reading it, so no content carries over between calls.
// Calls that overlap on the GPU (concurrent streams, or work queued by other host threads)
// race on the array and must not be issued.
#include <cuda_runtime.h>

#include <mutex>

#include "cib_common.cuh"
#include "rve.cuh"

// The work vectors r, p and Ap of the solve, one after the other.
static __device__ __align__(256) double g_pcg_work[3 * CIB_PCG_NOALLOC_MAX_VEC];

namespace cib {
namespace {

// Device address of g_pcg_work per device.  In host code the name g_pcg_work is only a
// host-side stand-in for the device symbol, so the real address is looked up with that
// device current.  The lookup is remembered together with the CUDA context it was made in
// (its unique context id): after cudaDeviceReset the device gets a new primary context, in
// which the library's module -- and the array -- may sit elsewhere, so a changed id makes
// the next call look the address up again (as does a driver without context ids, on every
// call).
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

struct WorkSlot {
  unsigned long long ctx_id;
  double* ptr;
};

std::mutex g_work_mutex;
WorkSlot g_work_slot[64] = {};

// Id of the calling thread's current context (0 when the driver entry points are missing).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) return 0;
  return id;
}

int work_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  if (dev < 0 || dev >= 64) return CIB_ERANGE;
  std::lock_guard<std::mutex> lock(g_work_mutex);
  const unsigned long long ctx = current_context_id();
  WorkSlot& slot = g_work_slot[dev];
  if (slot.ptr == nullptr || ctx == 0 || slot.ctx_id != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_pcg_work);
    if (e != cudaSuccess || p == nullptr) {
      last_cuda_error_slot() = (int)(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
      return CIB_ECUDA;
    }
    slot.ptr = static_cast<double*>(p);
    slot.ctx_id = current_context_id();
  }
  *out = slot.ptr;
  return CIB_OK;
}

template <typename T>
int solve(const cib_rve_batch& b, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off,
          const int32_t* active, int64_t vec_len, double* work, const double* rhs, const double* dinv, double* x,
          double rtol, int32_t maxit, int32_t* status, int32_t* iterations, double* rel, double* xnorm,
          cudaStream_t st) {
  RvePcgArgs<T> a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.phase = b.phase;
  a.mats = rve_phase_table<T>(b);
  a.ngp = rve_point_stride(b);
  a.tparam = static_cast<const T*>(b.tparam);
  a.tflag = b.tflag;
  a.sys_rve = sys_rve;
  a.sys_off = sys_off;
  a.active = active;
  a.b = rhs;
  a.dinv = dinv;
  a.x = x;
  a.r = work;
  a.p = work + vec_len;
  a.Ap = work + 2 * vec_len;
  a.rtol = rtol;
  a.maxit = maxit;
  a.status = status;
  a.iterations = iterations;
  a.rel_residual = rel;
  a.xnorm = xnorm;
  a.vec_len = vec_len;  // a system outside the work array is skipped with status 3
  return launch_rve_pcg<T>(a, nsys, b.max_nxy, st);
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_rve_pcg_noalloc(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve,
                                   const int64_t* sys_off, const int32_t* active, int64_t vec_len, const double* b,
                                   const double* dinv, double* x, double rtol, int32_t maxit, int32_t* status,
                                   int32_t* iterations, double* rel_residual, double* xnorm, void* stream) {
  if (!batch || batch->nrve < 0 || batch->nelem < 0 || batch->nphase < 1 || batch->nphase > RVE_MAX_PHASES || !batch->desc ||
      !batch->phase || (batch->precision != 32 && batch->precision != 64) || nsys < 0 || !sys_rve || !sys_off ||
      !b || !dinv || !x || !status || !iterations || !rel_residual || !xnorm || maxit < 0 || !batch->tparam ||
      !batch->tflag || batch->max_nxy <= 0 || vec_len < 0)
    return CIB_EINVAL;
  if (vec_len > CIB_PCG_NOALLOC_MAX_VEC) return CIB_ERANGE;  // the work array is too small for this call
  if (nsys == 0) return CIB_OK;
  double* work = nullptr;
  const int rc = work_address(&work);
  if (rc != CIB_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64 ? solve<double>(*batch, nsys, sys_rve, sys_off, active, vec_len, work, b, dinv, x,
                                                rtol, maxit, status, iterations, rel_residual, xnorm, st)
                                : solve<float>(*batch, nsys, sys_rve, sys_off, active, vec_len, work, b, dinv, x,
                                               rtol, maxit, status, iterations, rel_residual, xnorm, st);
}
