// des_shade_backward_noalloc: the fused adjoint with its scratch memory in a static device array.
//
// Who needs this: code that must not allocate device memory while it runs -- e.g. a renderer or
// simulator that hands this library device pointers from inside its own memory pool or real-time
// loop, where a cudaMalloc would synchronise the device, fragment a carefully sized pool, or is
// simply forbidden by the host framework.  Such a caller cannot provide the workspace that
// des_shade_backward asks for.  This entry point takes the same inputs and outputs and finds its
// scratch in `g_noalloc_scratch` below instead.
//
// Limits and behaviour:
//  * the array is DES_SHADE_NOALLOC_SCRATCH_BYTES (4 MiB) and lives as long as the library is loaded:
//    every GPU on which it is used keeps those 4 MiB until the process exits;
//  * when the array is too small for the default plan, the call runs in input order, and if need be
//    with the compact plan (DES_COMPACT: fewest persistent CTAs; same results, slower); a call
//    whose des_shade_workspace_bytes(P, H, W, flags | DES_COMPACT, 1, device) exceeds the array is
//    rejected with DES_ERR_WORKSPACE before anything is launched (on a 148-SM B200 this admits any
//    point count with env maps up to 16 x 32 texels, and larger maps only for small batches);
//  * all calls share the one array and it keeps the previous call's contents: the launch path resets
//    the tile counter and error word and overwrites the texel table and every env-gradient partial it
//    reads, so nothing left over is ever used -- but two calls whose work overlaps on the GPU (other
//    streams, other host threads) race on the array and corrupt each other's results;
//  * DES_REUSE_ORDER and DES_REUSE_TABLE are ignored here: no forward ever leaves its state in this array, so a
//    call that ordered its points always computes the ordering itself (a permutation left over from
//    an earlier call of another size would drop points);
//  * errors found on the device (out-of-range triangle or vertex ids, which des_workspace_status
//    reports for a caller-owned workspace) are not observable through this entry point: such points
//    shade to zero, as with the regular entry point, but the error word is not handed to the caller;
//  * the first call on each device looks up the array's device address with cudaGetSymbolAddress
//    (once per device, with that device current); that first call should be made before any CUDA
//    stream capture is started.
// It calls no cudaMalloc / cudaFree and no allocating library routine.
#include <cuda_runtime.h>

#include <mutex>

#include "diff_envshade_b200.h"

namespace {

// The scratch.  In host code this name is only a stand-in for the device symbol, not a device
// address; the address comes from cudaGetSymbolAddress in scratch_address() below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[DES_SHADE_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DES_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return DES_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return DES_ERR_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return DES_OK;
}

}  // namespace

extern "C" int des_shade_backward_noalloc(const des_shade_args* args, unsigned flags, const float* grad_shading,
                                          const float* grad_diffuse_shading, float* g_normal, float* g_view_dir,
                                          float* g_albedo, float* g_specular_albedo, float* g_roughness,
                                          float* g_envmap, des_stream_t stream) {
  if (args == nullptr) return DES_ERR_INVALID_ARGUMENT;
  flags &= ~(unsigned)(DES_REUSE_ORDER | DES_REUSE_TABLE);  // the array never holds a forward's state
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DES_ERR_CUDA;
  const size_t need = des_shade_workspace_bytes(args->P, args->H, args->W, flags | DES_COMPACT, 1, dev);
  if (need == 0) return args->C != 3 ? DES_ERR_UNSUPPORTED : DES_ERR_INVALID_ARGUMENT;
  if (need > sizeof(g_noalloc_scratch)) return DES_ERR_WORKSPACE;
  void* scratch = nullptr;
  const int st = scratch_address(&scratch);
  if (st != DES_OK) return st;
  return des_shade_backward(args, flags, grad_shading, grad_diffuse_shading, g_normal, g_view_dir, g_albedo,
                            g_specular_albedo, g_roughness, g_envmap, scratch, sizeof(g_noalloc_scratch), stream);
}
