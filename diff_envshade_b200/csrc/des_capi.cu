// C-ABI layer: argument validation and the reference-named entry points.
// Every function here is declared in include/diff_envshade_b200.h.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "des_internal.h"
#include "diff_envshade_b200.h"

namespace {

constexpr int64_t kMaxTexels = int64_t(1) << 24;

// Shape / pointer checks the reference leaves to the caller ("TODO: shape check",
// bruteforce_shader.cu:3289).  Returns DES_OK or the status to report.
int validate(const des_shade_args* a, unsigned flags, bool backward, const void* out0) {
  if (a == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if (a->C != 3) return DES_ERR_UNSUPPORTED;
  if (a->P < 0 || a->H <= 0 || a->W <= 0) return DES_ERR_INVALID_ARGUMENT;
  if ((int64_t)a->H * a->W > kMaxTexels) return DES_ERR_UNSUPPORTED;
  if (flags & ~(unsigned)(DES_DIFFUSE | DES_SPECULAR | DES_CLAMP | DES_INPUT_ORDER | DES_COMPACT | DES_REUSE_ORDER |
                          DES_REUSE_TABLE))
    return DES_ERR_INVALID_ARGUMENT;
  if (a->envmap == nullptr || a->light2obj_rotmat == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if (a->P == 0) return DES_OK;
  if (a->normal == nullptr || out0 == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if ((flags & DES_DIFFUSE) && a->albedo == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if ((flags & DES_SPECULAR) &&
      (a->view_dir == nullptr || a->specular_albedo == nullptr || a->roughness == nullptr))
    return DES_ERR_INVALID_ARGUMENT;
  if ((flags & DES_CLAMP) && a->view_dir == nullptr) return DES_ERR_INVALID_ARGUMENT;
  if (a->visibility != nullptr) {
    const int64_t need_slots = ((int64_t)a->H * a->W + 31) / 32;
    if (a->N_face <= 0 || a->N_vertex <= 0 || a->N_slot < need_slots) return DES_ERR_INVALID_ARGUMENT;
    if (a->face_vertex_list == nullptr || a->nearest_triangle_id == nullptr || a->barycentric_coord == nullptr)
      return DES_ERR_INVALID_ARGUMENT;
  }
  (void)backward;
  return DES_OK;
}

des_shade_args make_args(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal, const float* view_dir,
                         const float* albedo, const float* specular_albedo, const float* roughness,
                         const float* envmap, const float* R) {
  des_shade_args a{};
  a.P = P;
  a.H = H;
  a.W = W;
  a.C = C;
  a.normal = normal;
  a.view_dir = view_dir;
  a.albedo = albedo;
  a.specular_albedo = specular_albedo;
  a.roughness = roughness;
  a.envmap = envmap;
  a.light2obj_rotmat = R;
  return a;
}

}  // namespace

extern "C" {

const char* des_status_string(int status) {
  switch (status) {
    case DES_OK: return "ok";
    case DES_ERR_INVALID_ARGUMENT: return "invalid argument (null pointer, negative size or inconsistent shapes)";
    case DES_ERR_UNSUPPORTED: return "Channel number not supported! (only C == 3) or size beyond the supported range";
    case DES_ERR_WORKSPACE: return "workspace missing, not 256-byte aligned, or smaller than des_*_workspace_bytes";
    case DES_ERR_CUDA: return "CUDA runtime error";
    case DES_ERR_BAD_INDEX: return "triangle or vertex index out of range in visibility inputs";
    case DES_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
  }
}

int des_abi_version(void) { return 1; }

size_t des_shade_workspace_bytes(int64_t P, int32_t H, int32_t W, unsigned flags, int backward, int device) {
  if (P < 0 || H <= 0 || W <= 0 || (int64_t)H * W > kMaxTexels) return 0;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return 0;
  if (device != prev && cudaSetDevice(device) != cudaSuccess) return 0;
  des::LaunchPlan lp = des::plan_launch(P, H, W, backward != 0, device, (flags & DES_COMPACT) != 0);
  if (flags & DES_INPUT_ORDER) {
    lp.sort = false;
    lp.sort_chunks = 0;
  }
  int grid = std::max(des::shade_grid(lp, flags, backward != 0, false), des::shade_grid(lp, flags, backward != 0, true));
  if (device != prev) cudaSetDevice(prev);
  if (grid <= 0) return 0;
  return des::workspace_bytes(lp, backward != 0, grid);
}

int des_shade_forward(const des_shade_args* args, unsigned flags, float* shading, float* diffuse_shading,
                      void* workspace, size_t workspace_bytes, des_stream_t stream) {
  int st = validate(args, flags, false, shading);
  if (st != DES_OK) return st;
  des::ShadeCall c{};
  c.args = args;
  c.flags = flags;
  c.backward = false;
  c.shading = shading;
  c.white = diffuse_shading;
  c.workspace = workspace;
  c.workspace_bytes = workspace_bytes;
  return des::launch_shade(c, stream);
}

int des_shade_backward(const des_shade_args* args, unsigned flags, const float* grad_shading,
                       const float* grad_diffuse_shading, float* g_normal, float* g_view_dir, float* g_albedo,
                       float* g_specular_albedo, float* g_roughness, float* g_envmap, void* workspace,
                       size_t workspace_bytes, des_stream_t stream) {
  int st = validate(args, flags, true, g_normal);
  if (st != DES_OK) return st;
  if (args->P > 0 && grad_shading == nullptr) return DES_ERR_INVALID_ARGUMENT;
  des::ShadeCall c{};
  c.args = args;
  c.flags = flags;
  c.backward = true;
  c.g_shading = grad_shading;
  c.g_white = grad_diffuse_shading;
  c.g_normal = g_normal;
  c.g_view = g_view_dir;
  c.g_albedo = g_albedo;
  c.g_spec = g_specular_albedo;
  c.g_rough = g_roughness;
  c.g_envmap = g_envmap;
  c.workspace = workspace;
  c.workspace_bytes = workspace_bytes;
  return des::launch_shade(c, stream);
}

size_t des_relight_workspace_bytes(int64_t P, int32_t H, int32_t W, int32_t K) {
  if ((int64_t)H * W > kMaxTexels) return 0;
  return des::relight_workspace_bytes(P, H, W, K);
}

int des_relight_multienv(const des_shade_args* args, const float* envmaps, int32_t K, unsigned flags, float* out,
                         void* workspace, size_t workspace_bytes, des_stream_t stream) {
  if (args == nullptr || envmaps == nullptr || K <= 0) return DES_ERR_INVALID_ARGUMENT;
  des_shade_args a = *args;
  a.envmap = envmaps;  // validated like a single map; the relight path reads all K of them
  int st = validate(&a, flags & ~(unsigned)DES_RELIGHT_BF16, false, out);
  if (st != DES_OK) return st;
  return des::launch_relight(a, envmaps, K, flags, out, workspace, workspace_bytes,
                             reinterpret_cast<cudaStream_t>(stream));
}

int des_texel_table(int32_t H, int32_t W, const float* light2obj_rotmat, float* table_out, des_stream_t stream) {
  if (H <= 0 || W <= 0 || (int64_t)H * W > kMaxTexels || light2obj_rotmat == nullptr || table_out == nullptr)
    return DES_ERR_INVALID_ARGUMENT;
  return des::launch_texel_table(H, W, light2obj_rotmat, table_out, stream);
}

int des_set_timing_events(void* start_event, void* stop_event) {
  des::set_timing_events(static_cast<cudaEvent_t>(start_event), static_cast<cudaEvent_t>(stop_event));
  return DES_OK;
}

unsigned long long des_kernel_launches(void) { return des::launches_so_far(); }

int des_workspace_status(void* workspace, size_t workspace_bytes, int* status_out, des_stream_t stream) {
  if (workspace == nullptr || workspace_bytes < des::kCtrlBytes || status_out == nullptr)
    return DES_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned* ctrl = static_cast<unsigned*>(workspace);
  unsigned err = 0;
  if (cudaMemcpyAsync(&err, ctrl + des::kCtrlError, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return DES_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return DES_ERR_CUDA;
  if (cudaMemsetAsync(ctrl + des::kCtrlError, 0, sizeof(unsigned), s) != cudaSuccess) return DES_ERR_CUDA;
  *status_out = (err & 2u) ? DES_ERR_TIMEOUT : (err ? DES_ERR_BAD_INDEX : DES_OK);
  return DES_OK;
}

// ---------------------------------------------------------------------------------------------
// Reference-named entry points
// ---------------------------------------------------------------------------------------------

int des_bruteforce_diffuse_shader_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                          const float* albedo, const float* envmap, const float* light2obj_rotmat,
                                          float* shading, void* workspace, size_t workspace_bytes,
                                          des_stream_t stream) {
  des_shade_args a = make_args(P, H, W, C, normal, nullptr, albedo, nullptr, nullptr, envmap, light2obj_rotmat);
  return des_shade_forward(&a, DES_DIFFUSE, shading, nullptr, workspace, workspace_bytes, stream);
}

int des_bruteforce_diffuse_shader_backward(int64_t P, int32_t H, int32_t W, int32_t C, const float* grad_shading,
                                           const float* normal, const float* albedo, const float* envmap,
                                           const float* light2obj_rotmat, float* grad_normal, float* grad_albedo,
                                           float* grad_envmap, void* workspace, size_t workspace_bytes,
                                           des_stream_t stream) {
  des_shade_args a = make_args(P, H, W, C, normal, nullptr, albedo, nullptr, nullptr, envmap, light2obj_rotmat);
  return des_shade_backward(&a, DES_DIFFUSE, grad_shading, nullptr, grad_normal, nullptr, grad_albedo, nullptr,
                            nullptr, grad_envmap, workspace, workspace_bytes, stream);
}

int des_bruteforce_specular_shader_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                           const float* view_dir, const float* albedo,
                                           const float* specular_albedo, const float* roughness,
                                           const float* envmap, const float* light2obj_rotmat, int enable_diffuse,
                                           int enable_specular, int clamp, float* shading, void* workspace,
                                           size_t workspace_bytes, des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  unsigned f = (enable_diffuse ? DES_DIFFUSE : 0u) | (enable_specular ? DES_SPECULAR : 0u) | (clamp ? DES_CLAMP : 0u);
  return des_shade_forward(&a, f, shading, nullptr, workspace, workspace_bytes, stream);
}

int des_bruteforce_specular_shader_backward(int64_t P, int32_t H, int32_t W, int32_t C, const float* grad_shading,
                                            const float* normal, const float* view_dir, const float* albedo,
                                            const float* specular_albedo, const float* roughness,
                                            const float* envmap, const float* light2obj_rotmat,
                                            int enable_diffuse, int enable_specular, int clamp,
                                            float* grad_normal, float* grad_view_dir, float* grad_albedo,
                                            float* grad_specular_albedo, float* grad_roughness,
                                            float* grad_envmap, void* workspace, size_t workspace_bytes,
                                            des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  unsigned f = (enable_diffuse ? DES_DIFFUSE : 0u) | (enable_specular ? DES_SPECULAR : 0u) | (clamp ? DES_CLAMP : 0u);
  return des_shade_backward(&a, f, grad_shading, nullptr, grad_normal, grad_view_dir, grad_albedo,
                            grad_specular_albedo, grad_roughness, grad_envmap, workspace, workspace_bytes, stream);
}

int des_bruteforce_specular_shader_forward2(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                            const float* view_dir, const float* albedo,
                                            const float* specular_albedo, const float* roughness,
                                            const float* envmap, const float* light2obj_rotmat,
                                            int enable_specular, float* shading, float* diffuse_shading,
                                            void* workspace, size_t workspace_bytes, des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  unsigned f = DES_DIFFUSE | (enable_specular ? DES_SPECULAR : 0u);
  return des_shade_forward(&a, f, shading, diffuse_shading, workspace, workspace_bytes, stream);
}

int des_bruteforce_specular_shader_backward2(int64_t P, int32_t H, int32_t W, int32_t C,
                                             const float* grad_shading, const float* grad_diffuse_shading,
                                             const float* normal, const float* view_dir, const float* albedo,
                                             const float* specular_albedo, const float* roughness,
                                             const float* envmap, const float* light2obj_rotmat,
                                             int enable_specular, float* grad_normal, float* grad_view_dir,
                                             float* grad_albedo, float* grad_specular_albedo,
                                             float* grad_roughness, float* grad_envmap, void* workspace,
                                             size_t workspace_bytes, des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  unsigned f = DES_DIFFUSE | (enable_specular ? DES_SPECULAR : 0u);
  return des_shade_backward(&a, f, grad_shading, grad_diffuse_shading, grad_normal, grad_view_dir, grad_albedo,
                            grad_specular_albedo, grad_roughness, grad_envmap, workspace, workspace_bytes, stream);
}

int des_bruteforce_specularvisibility_shader_forward2(
    int64_t P, int32_t H, int32_t W, int32_t C, int32_t N_face, int32_t N_vertex, int32_t N_slot,
    const float* normal, const float* view_dir, const float* albedo, const float* specular_albedo,
    const float* roughness, const float* envmap, const float* light2obj_rotmat, const int32_t* face_vertex_list,
    const int64_t* nearest_triangle_id, const float* barycentric_coord, const int32_t* visibility,
    int enable_specular, float* shading, float* diffuse_shading, void* workspace, size_t workspace_bytes,
    des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  a.N_face = N_face;
  a.N_vertex = N_vertex;
  a.N_slot = N_slot;
  a.face_vertex_list = face_vertex_list;
  a.nearest_triangle_id = nearest_triangle_id;
  a.barycentric_coord = barycentric_coord;
  a.visibility = reinterpret_cast<const uint32_t*>(visibility);
  if (visibility == nullptr) return DES_ERR_INVALID_ARGUMENT;
  unsigned f = DES_DIFFUSE | (enable_specular ? DES_SPECULAR : 0u);
  return des_shade_forward(&a, f, shading, diffuse_shading, workspace, workspace_bytes, stream);
}

int des_bruteforce_specularvisibility_shader_backward2(
    int64_t P, int32_t H, int32_t W, int32_t C, int32_t N_face, int32_t N_vertex, int32_t N_slot,
    const float* grad_shading, const float* grad_diffuse_shading, const float* normal, const float* view_dir,
    const float* albedo, const float* specular_albedo, const float* roughness, const float* envmap,
    const float* light2obj_rotmat, const int32_t* face_vertex_list, const int64_t* nearest_triangle_id,
    const float* barycentric_coord, const int32_t* visibility, int enable_specular, float* grad_normal,
    float* grad_view_dir, float* grad_albedo, float* grad_specular_albedo, float* grad_roughness,
    float* grad_envmap, void* workspace, size_t workspace_bytes, des_stream_t stream) {
  des_shade_args a =
      make_args(P, H, W, C, normal, view_dir, albedo, specular_albedo, roughness, envmap, light2obj_rotmat);
  a.N_face = N_face;
  a.N_vertex = N_vertex;
  a.N_slot = N_slot;
  a.face_vertex_list = face_vertex_list;
  a.nearest_triangle_id = nearest_triangle_id;
  a.barycentric_coord = barycentric_coord;
  a.visibility = reinterpret_cast<const uint32_t*>(visibility);
  if (visibility == nullptr) return DES_ERR_INVALID_ARGUMENT;
  unsigned f = DES_DIFFUSE | (enable_specular ? DES_SPECULAR : 0u);
  return des_shade_backward(&a, f, grad_shading, grad_diffuse_shading, grad_normal, grad_view_dir, grad_albedo,
                            grad_specular_albedo, grad_roughness, grad_envmap, workspace, workspace_bytes, stream);
}

}  // extern "C"
