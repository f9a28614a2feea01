// qcuDslashNoAlloc: the hopping term of qcuDslash without any device memory
// allocation in the call.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree while they run -
// a host framework that has already claimed the GPU's memory with its own
// pool allocator (so a foreign cudaMalloc fails or fragments its pool), or a
// time-critical loop that cannot afford the implicit device synchronisation
// that cudaMalloc/cudaFree bring. qcuDslash allocates its internal-layout
// staging fields on first use (and again when the lattice changes); this
// variant uses a fixed scratch array compiled into the library instead.
//
// Scratch: one file-scope __device__ array of kNoAllocMaxVh * 2 * 192 bytes
// (6 MiB): the input half spinor and the output half spinor in the internal
// FP64 layout. Every GPU that loads the library holds it until the process
// exits. Lattices whose half volume (rounded up to 32 sites) exceeds
// kNoAllocMaxVh = 16384 sites are rejected with QCU_ERR_INVALID_ARG.
//
// All calls share the one array, which keeps the last call's contents; every
// call overwrites the parts it reads before reading them (nothing has to start
// at zero). Calls whose work overlaps on the GPU - from two host threads, or
// two contexts on different streams of the same device - race on the array.
//
// Set-up, once per device and with that device current: the device address of
// the array is looked up with cudaGetSymbolAddress, and the code of the
// kernels the entry point launches is loaded (under lazy module loading a
// module, the array's included, is loaded and its device memory taken at
// first use). qcuContextCreate runs this set-up, so the 6 MiB are taken when
// the first context is created on a device and a call takes no device memory
// at all. Should that set-up fail there, the first call retries it (and then
// it may load code), so a context that is to be used under stream capture
// should make one call first. Host code must never hand the array's host-side
// name to a kernel.
//
// The address is cached per device for the life of the process: after a
// cudaDeviceReset (or a reset of the primary context) every context of this
// library is invalid anyway, and neither it nor this entry point may be used
// again in that process.
#include <string.h>

#include <mutex>
#include <string>

#include "qcu_context.h"

namespace qcu {

constexpr int kNoAllocMaxVh = 16384;
constexpr int kNoAllocMaxDevices = 64;

// [0, Vh_pad*12): input (double2 chunks), [Vh_pad*12, 2*Vh_pad*12): output
static __device__ __align__(256) double2 g_noalloc_scratch[2 * kNoAllocMaxVh * 12];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

typedef void (*DslashKernelFn)(const DslashArgs);
DslashKernelFn pick_f64(bool dag, int epi, int fin);

static int noalloc_lookup(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    set_error(QCU_ERR_UNSUPPORTED, "device index beyond the no-alloc scratch table");
    return QCU_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // device `device` is current
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    // the kernels of a call: AoS -> internal, the FP64 hop (D and D^dag),
    // internal -> AoS
    e = preload_spinor_io_f64();
    cudaFuncAttributes fa;
    for (int dag = 0; dag < 2 && e == cudaSuccess; dag++) {
      DslashKernelFn fn = pick_f64(dag != 0, 0, FIN_NONE);
      e = fn ? cudaFuncGetAttributes(&fa, fn) : cudaErrorInvalidDeviceFunction;
    }
    if (e != cudaSuccess) return cuda_status(e, "loading the no-alloc kernels");
    g_noalloc_addr[device] = p;
  }
  return QCU_SUCCESS;
}

int noalloc_prepare(int device) { return noalloc_lookup(device); }

static int noalloc_scratch(int device, double2** out) {
  QCU_CHECK(noalloc_lookup(device));
  *out = static_cast<double2*>(g_noalloc_addr[device]);
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

extern "C" int qcuDslashNoAlloc(qcu_context ctx, void* out, const void* in, int parity, int dagger, double bc_t) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));  // makes ctx->device current
  const Geom& g = ctx->g;
  if (g.Vh_pad > kNoAllocMaxVh) {
    set_error(QCU_ERR_INVALID_ARG, "qcuDslashNoAlloc: half volume " + std::to_string(g.Vh) +
                                       " exceeds its fixed scratch of 16384 sites per parity");
    return QCU_ERR_INVALID_ARG;
  }
  if (!out || !in || (parity != 0 && parity != 1)) {
    set_error(QCU_ERR_INVALID_ARG, "bad dslash arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!is_device_ptr_on(out, ctx->device) || !is_device_ptr_on(in, ctx->device)) {
    set_error(QCU_ERR_INVALID_ARG,
              "qcuDslashNoAlloc takes device pointers of the context's GPU only (host data would need staging)");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  double2* scratch = nullptr;
  QCU_CHECK(noalloc_scratch(ctx->device, &scratch));
  SpinorView vin{scratch, nullptr, 1};
  SpinorView vout{scratch + (size_t)g.Vh_pad * 12, nullptr, 1};
  QCU_CHECK_CUDA(launch_spinor_in(PREC_DOUBLE, g, 1, in, 0, vin, ctx->stream));
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.g = g;
  a.parity = parity;
  a.nrhs = 1;
  a.in = CSpinorView(vin);
  a.out = vout;
  a.gauge = ctx_gauge(ctx, PREC_DOUBLE);
  a.bc_t = bc_t;
  QCU_CHECK_CUDA(launch_dslash(PREC_DOUBLE, dagger != 0, 0, FIN_NONE, a, ctx->shape1, ctx->stream));
  QCU_CHECK_CUDA(launch_spinor_out(PREC_DOUBLE, g, 1, CSpinorView(vout), out, 0, ctx->stream));
  ctx->launches += 3;
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}
