// Internal declarations shared by the kernel translation units and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <utility>

#include "diff_envshade_b200.h"

namespace des {

constexpr int kMaxThreads = 512;  // largest CTA of the shading kernels (16 warps)
constexpr int kChunk = 2048;      // texels of the table staged in shared memory at once
constexpr size_t kCtrlBytes = 256;
// Normal-direction ordering of the points (calls with P >= kSortMinP): a stable counting sort by
// the octahedral cell (32 x 32 cells, Morton order) of each normal, in chunks of kSortChunk points.
constexpr int kSortBins = 1024;
constexpr int kSortThreads = 512;       // threads of a ranking CTA (16 warps, 64 points each per pass)
constexpr int kSortMinChunk = 1024;     // points ranked by one CTA: the smallest power-of-two
constexpr int kSortMaxChunks = 128;     //   multiple of 1024 that needs at most 128 CTAs
constexpr int64_t kSortMinP = 16384;
constexpr int64_t kSortMaxP = int64_t(1) << 24;  // per-warp 16-bit cell counters stay below 2^16
inline int sort_chunk_for(int64_t P) {
  int chunk = kSortMinChunk;
  while ((int64_t)chunk * kSortMaxChunks < P) chunk *= 2;
  return chunk;
}

// Programmatic dependent launch (sm_90+): every kernel launched with launch_pdl() starts with
// pdl_enter(), which lets the next kernel in its stream be scheduled as soon as all of its own CTAs
// are running (launch_dependents; the next kernel can only be launched once every CTA of this one
// has started, so a waiting kernel never holds the resources a running one still needs), then
// waits until its predecessor has completed and its writes are visible (wait) before it touches
// global memory.  The next kernel's launch and CTA start-up overlap this kernel's tail; a
// predecessor that does not take part (any other kernel in the stream) simply completes first, as
// without the attribute.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
#endif

// Launches `kernel` on (grid, block, smem, stream) with programmatic stream serialization.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// control words at the start of every workspace
// (the forward and the adjoint claim tiles from separate counters, so an adjoint that reuses the
// texel table of the forward before it -- DES_REUSE_TABLE -- needs no kernel to reset its counter;
// every table or ordering kernel resets all three words)
enum : int { kCtrlTileCounter = 0, kCtrlError = 1, kCtrlTileCounterBwd = 2 };

// Kernel parameters (passed by value in the launch).
struct ShadeParams {
  int64_t P;
  int HWpad, chunk, ntiles;
  int N_face, N_vertex;
  const float* normal;
  const float* view;
  const float* albedo;
  const float* spec;
  const float* rough;
  const int32_t* faces;
  const int64_t* tri;
  const float* bary;
  const uint32_t* vis;
  const int32_t* perm;   // optional: tile slot -> point index (normal-direction order)
  const float4* table;  // [HWpad][2] texel records
  bool clamp;
  bool env_in_smem;
  unsigned* ctrl;
  // forward outputs
  float* shading;
  float* white;
  // backward inputs / outputs
  const float* g_shading;
  const float* g_white;
  float* g_normal;
  float* g_view;
  float* g_albedo;
  float* g_spec;
  float* g_rough;
  double* env_partial;  // [grid][3][HWpad]
};

struct LaunchPlan {
  int HWpad, chunk, ntiles, nw;
  bool env_in_smem;
  bool sort;        // order the points by normal direction first
  int sort_chunk;   // points per ranking CTA
  int sort_chunks;  // ceil(P / sort_chunk) when sorting
  size_t smem;
  int sms, max_smem;
};

struct ShadeCall {
  const des_shade_args* args;
  unsigned flags;
  bool backward;
  float* shading;
  float* white;
  const float* g_shading;
  const float* g_white;
  float* g_normal;
  float* g_view;
  float* g_albedo;
  float* g_spec;
  float* g_rough;
  float* g_envmap;
  void* workspace;
  size_t workspace_bytes;
};

// compact: the plan with the smallest workspace: input order, and for the adjoint the widest CTAs
// (fewest persistent CTAs, so fewest env-map gradient partials).
LaunchPlan plan_launch(int64_t P, int H, int W, bool backward, int dev, bool compact = false);
size_t workspace_bytes(const LaunchPlan& lp, bool backward, int grid);
int shade_grid(const LaunchPlan& lp, unsigned flags, bool backward, bool vis);
int launch_shade(const ShadeCall& call, des_stream_t stream);
int launch_texel_table(int H, int W, const float* R, float* out, des_stream_t stream);
// Texel records (see des_table_kernel) for an env map; also resets the workspace control words.
int launch_table(int H, int W, int HWpad, const float* R, const float* env, float4* rec, unsigned* ctrl,
                 cudaStream_t stream);
void set_timing_events(cudaEvent_t start, cudaEvent_t stop);
// The events set by set_timing_events (both null when timing is off).
void timing_events(cudaEvent_t& start, cudaEvent_t& stop);
// Normal-direction ordering of P points on its own (kSortMinP..kSortMaxP points): perm[P] receives
// the point indices in the order the shading kernels use; scratch needs point_order_scratch_bytes(P).
size_t point_order_scratch_bytes(int64_t P);
int launch_point_order(const float* normal, int64_t P, void* scratch, int32_t* perm, cudaStream_t stream);
// Running count of kernel launches issued by this library (all streams and devices).
void count_launches(int n);
unsigned long long launches_so_far();
size_t relight_workspace_bytes(int64_t P, int H, int W, int K);
int launch_relight(const des_shade_args& a, const float* envmaps, int K, unsigned flags, float* out, void* ws,
                   size_t ws_bytes, cudaStream_t stream);

}  // namespace des
