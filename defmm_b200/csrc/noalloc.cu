// Direct sums without any device allocation (defmm_direct_noalloc).
//
// Who needs this: callers that must not call cudaMalloc / cudaFree at the
// point where they check potentials -- applications whose framework owns all
// device memory through its own pool and forbids side allocations, and
// latency-bound loops that cannot afford the device-wide synchronisation
// cudaFree implies.  The regular check (defmm_check_full) allocates a scratch
// buffer for its samples; this entry point keeps its scratch in a file-scope
// device array instead, so a call allocates nothing.  The first call on a
// device looks up the array's address (cudaGetSymbolAddress, which may load
// this file's device code); make that call before any stream capture.  The
// call reads the charges of the handle's last host gemv on the caller's
// stream; the handle's next host gemv waits for that read (an event) before
// it overwrites them.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents.  Calls that overlap on the GPU (two streams, two threads,
// or two handles on one device at the same time) race on it: serialise them.
#include <mutex>
#include <string>

#include "../../include/defmm_b200.h"
#include "engine_internal.h"

namespace {

// Split-source partial sums: nt targets x S source chunks, complex FP64.
constexpr int64_t kScratchElems = 262144;  // 4 MiB
static __device__ __align__(256) double2 g_direct_scratch[kScratchElems];

constexpr int kTPB = 128;  // targets per CTA (one per thread)
constexpr int kTile = 256; // sources staged in shared memory per step

// partial[s * nt + t] = sum over source chunk s of q_j G(x_t, y_j): the
// reference's CheckFULL / P2P arithmetic (include/interface.hpp:178-221,
// include/operators/P2P.hpp:43-79), FP64; pairs with |x - y|^2 < 1e-16
// (|x - y| < 1e-8) contribute zero, as in the reference's CheckFULL.  Every
// (s, t < nt) entry is written, empty chunks included, so nothing in the
// scratch needs clearing first.
__global__ void __launch_bounds__(kTPB) k_direct_partial(int64_t ns, const double* __restrict__ spos,
                                                         const int32_t* __restrict__ sperm,
                                                         const double2* __restrict__ qin, int64_t nt,
                                                         const double* __restrict__ tpos, double kappa, int S,
                                                         double2* __restrict__ partial) {
  __shared__ double sx[kTile], sy[kTile], sz[kTile];
  __shared__ double2 sq[kTile];
  const int64_t t = (int64_t)blockIdx.x * kTPB + threadIdx.x;
  const int s = blockIdx.y;
  const int64_t j0 = ns * s / S, j1 = ns * (s + 1) / S;
  const bool act = t < nt;
  double x0 = 0., x1 = 0., x2 = 0.;
  if (act) {
    x0 = tpos[3 * t];
    x1 = tpos[3 * t + 1];
    x2 = tpos[3 * t + 2];
  }
  const double pi4m1 = 1. / (4. * 3.14159265358979323846);
  double pr = 0., pim = 0.;
  for (int64_t b = j0; b < j1; b += kTile) {
    const int n = (int)min((int64_t)kTile, j1 - b);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kTPB) {
      const int64_t j = b + i;
      sx[i] = spos[3 * j];
      sy[i] = spos[3 * j + 1];
      sz[i] = spos[3 * j + 2];
      sq[i] = qin[sperm[j]];
    }
    __syncthreads();
    if (act) {
      for (int i = 0; i < n; i++) {
        const double dx = x0 - sx[i], dy = x1 - sy[i], dz = x2 - sz[i];
        const double R = dx * dx + dy * dy + dz * dz;
        if (R < 1.e-16) continue;
        double K = 1. / sqrt(R);
        const double rr = K * R * kappa;
        K *= pi4m1;
        double sn, cs;
        sincos(rr, &sn, &cs);
        pr += cs * K * sq[i].x - sn * K * sq[i].y;
        pim += cs * K * sq[i].y + sn * K * sq[i].x;
      }
    }
  }
  if (act) partial[(int64_t)s * nt + t] = make_double2(pr, pim);
}

// out[t] = sum_s partial[s * nt + t], chunks in order (deterministic).
__global__ void k_direct_reduce(int64_t nt, int S, const double2* __restrict__ partial, double2* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double2 a = partial[t];
  for (int s = 1; s < S; s++) {
    const double2 b = partial[(int64_t)s * nt + t];
    a.x += b.x;
    a.y += b.y;
  }
  out[t] = a;
}

// Device address of the scratch array, per device (host code may not pass
// the symbol itself to a kernel: it names a host-side stand-in).  Outside
// stream capture the address is looked up on every call, which costs a table
// lookup once the module is loaded and stays right after a device reset
// reloads it; inside a capture the address of the last uncaptured call on
// that device is used, so a call must precede any capture.
std::mutex g_mu;
void* g_addr[64] = {nullptr};

int scratch_address(int dev, bool capturing, double2** out, std::string& err) {
  if (dev < 0 || dev >= 64) {
    err = "device index out of range";
    return DEFMM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!capturing) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return DEFMM_ERR_CUDA;
    }
    g_addr[dev] = p;
  } else if (!g_addr[dev]) {
    err = "defmm_direct_noalloc: the first call on a device must come before any stream capture";
    return DEFMM_ERR_ARG;
  }
  *out = static_cast<double2*>(g_addr[dev]);
  return 0;
}

// The calling thread's current device, put back on every return.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int defmm_direct_noalloc(defmm_handle* h, const double* d_targets, int64_t nt, double* d_out,
                                    void* stream) {
  if (!h || !d_targets || !d_out || nt < 1) return DEFMM_ERR_ARG;
  dfb::HandleView v;
  int st = dfb::handle_view(h, &v);
  if (st) return st;
  if (nt > kScratchElems)
    return dfb::handle_fail(h, DEFMM_ERR_ARG,
                            "defmm_direct_noalloc: at most 262144 targets per call (scratch of 4 MiB)");
  DeviceGuard guard;
  cudaError_t e = cudaSetDevice(v.device);
  if (e != cudaSuccess) return dfb::handle_fail(h, DEFMM_ERR_CUDA, cudaGetErrorString(e));
  cudaStream_t s = stream ? (cudaStream_t)stream : v.stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return dfb::handle_fail(h, DEFMM_ERR_CUDA, cudaGetErrorString(e));
  std::string msg;
  double2* partial = nullptr;
  st = scratch_address(v.device, cap != cudaStreamCaptureStatusNone, &partial, msg);
  if (st) return dfb::handle_fail(h, st, msg.c_str());
  // as many source chunks as the scratch holds (<= 64), at most one per 1024 sources
  int64_t S = kScratchElems / nt;
  S = S < 64 ? S : 64;
  const int64_t Smax = (v.nS + 1023) / 1024;
  S = S < Smax ? S : Smax;
  if (S < 1) S = 1;
  dim3 grid((unsigned)((nt + kTPB - 1) / kTPB), (unsigned)S);
  k_direct_partial<<<grid, kTPB, 0, s>>>(v.nS, v.S_pos, v.S_perm, v.qin, nt, d_targets, v.kappa, (int)S, partial);
  k_direct_reduce<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(nt, (int)S, partial, reinterpret_cast<double2*>(d_out));
  e = cudaGetLastError();
  if (e != cudaSuccess) return dfb::handle_fail(h, DEFMM_ERR_CUDA, cudaGetErrorString(e));
  // the handle's next host gemv overwrites the charges read here: it waits
  // for this event first
  e = cudaEventRecord(v.qin_read, s);
  if (e != cudaSuccess) return dfb::handle_fail(h, DEFMM_ERR_CUDA, cudaGetErrorString(e));
  return 0;
}
