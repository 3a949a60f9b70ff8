/*
 * diff_envshade_b200 -- C ABI of the B200 (sm_100a) environment-map shading kernels.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t, returns a
 * des_status (0 = DES_OK), launches asynchronously on the given stream, and allocates
 * nothing: scratch memory is passed in by the caller (size from des_*_workspace_bytes).
 *
 * Tensor layouts are the reference extension's (zjumsj/diff_envshade, gsface_shader.h:64-118):
 *   normal, view_dir, albedo, specular_albedo   P x 3 float32, row-major (AoS)
 *   roughness                                   P x 1 float32
 *   envmap                                      C x H x W float32, planar, row 0 = top
 *   light2obj_rotmat                            3 x 3 float32 row-major, l' = R l
 *   face_vertex_list                            3 x N_face int32 (SoA)
 *   nearest_triangle_id                         P int64
 *   barycentric_coord                           3 x P float32 (SoA)
 *   visibility                                  N_slot x N_vertex 32-bit words; texel t = row*W + col
 *                                               is bit (t % 32) of visibility[t / 32][vertex]
 * Only C == 3 is supported (as in the reference, bruteforce_shader.cu:3332).
 */
#ifndef DIFF_ENVSHADE_B200_H_
#define DIFF_ENVSHADE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* des_stream_t; /* a cudaStream_t; NULL = legacy default stream */

typedef enum des_status {
  DES_OK = 0,
  DES_ERR_INVALID_ARGUMENT = 1, /* a null pointer, negative size, or shapes that do not fit together */
  DES_ERR_UNSUPPORTED = 2,      /* e.g. C != 3 ("Channel number not supported!") */
  DES_ERR_WORKSPACE = 3,        /* workspace pointer null, misaligned or too small */
  DES_ERR_CUDA = 4,             /* a CUDA runtime call or kernel launch failed */
  DES_ERR_BAD_INDEX = 5,        /* a triangle or vertex id outside its table was seen on the device */
  DES_ERR_TIMEOUT = 6           /* a bounded device-side wait ran out (serving queue) */
} des_status;

/* Shading-term switches for des_shade_forward / des_shade_backward. */
#define DES_DIFFUSE 1u  /* Lambert term                                                 */
#define DES_SPECULAR 2u /* GGX term (Schlick Fresnel, Schlick-Smith G, GGX NDF)          */
#define DES_CLAMP 4u    /* backface clamp: a point with n.v <= 0 shades to zero          */
#define DES_RELIGHT_BF16 8u /* des_relight_multienv: plain BF16 operands (default: BF16 hi+lo split) */
/* des_shade_*: shade the points in input order.  By default calls with P >= 16384 first order the
 * points by the octahedral cell of their normal, so that a warp's 32 points face the same way and
 * texels below all of their horizons are skipped.  The outputs are the same either way (per-point
 * values bit for bit; the env-map gradient up to FP64 summation order).  Input order needs a
 * smaller workspace; a workspace too small for the ordering also falls back to input order. */
#define DES_INPUT_ORDER 16u
/* des_shade_*: the smallest workspace -- input order, and for the adjoint the widest CTAs (the
 * fewest persistent CTAs, each of which keeps its own FP64 env-map gradient partial).  Slower.  The
 * forward's outputs are the same bit for bit; the adjoint's agree to FP32 rounding (each point's
 * texel sum is split over a different number of warps).  A workspace too small for the default
 * plan also falls back to input order, then to this plan. */
#define DES_COMPACT 32u
/* des_shade_*: the workspace already holds the point ordering of these same normals (same P, H, W)
 * from the previous call made with it -- typically the forward of the adjoint that follows -- so the
 * ordering kernels are skipped.  Only the caller can know this: the workspace must not have been
 * used for anything else in between (a damaged permutation loses points; entries out of range
 * are skipped and reported as DES_ERR_BAD_INDEX by des_workspace_status).  If only the normals'
 * values changed, the stale ordering is still a valid permutation: per-point outputs are the same
 * bit for bit and the env-map gradient differs only in FP64 summation order.  Ignored for calls
 * that do not order their points. */
#define DES_REUSE_ORDER 64u
/* des_shade_backward: the call immediately before this one on the same workspace was the forward
 * of the same problem (same env map and rotation, and for an ordered call the same normals, with
 * DES_REUSE_ORDER also passed): its texel table is reused and the adjoint launches no table or
 * ordering kernel first.  Only the caller can know this; the table kernel's reset of the error word
 * is skipped too, so des_workspace_status then reports the forward's and the adjoint's errors
 * together.  Ignored by des_shade_forward. */
#define DES_REUSE_TABLE 128u

/* All inputs of one shading call.  The visibility block is ignored when visibility == NULL. */
typedef struct des_shade_args {
  int64_t P;
  int32_t H, W, C;
  const float* normal;
  const float* view_dir;        /* may be NULL when neither DES_SPECULAR nor DES_CLAMP is set */
  const float* albedo;          /* may be NULL when DES_DIFFUSE is not set                    */
  const float* specular_albedo; /* may be NULL when DES_SPECULAR is not set                   */
  const float* roughness;       /* may be NULL when DES_SPECULAR is not set                   */
  const float* envmap;
  const float* light2obj_rotmat;
  int32_t N_face, N_vertex, N_slot;
  const int32_t* face_vertex_list;
  const int64_t* nearest_triangle_id;
  const float* barycentric_coord;
  const uint32_t* visibility;   /* NULL = no visibility term */
} des_shade_args;

/* Human-readable text of a status code (static storage). */
const char* des_status_string(int status);

/* ABI version of this header (bumped on any signature change). */
int des_abi_version(void);

/* ---------------------------------------------------------------------------------------
 * Generic entry points
 * ------------------------------------------------------------------------------------- */

/* Scratch bytes des_shade_forward (backward = 0) or des_shade_backward (backward = 1) needs for
 * these sizes on `device`.  Returns 0 on an invalid argument. */
size_t des_shade_workspace_bytes(int64_t P, int32_t H, int32_t W, unsigned flags, int backward, int device);

/* shading[P x 3] = sum over texels of L * (albedo * diffuse weight + specular_albedo * GGX weight);
 * diffuse_shading[P x 3] (optional, may be NULL) = the same diffuse sum with a white albedo.
 * Replaces the kernels behind bruteforce_{diffuse,specular,specular_shader_clamp}_*forward* and
 * bruteforce_specular{,visibility}_shader_forward2 (reference bruteforce_shader.cu:2687-3336). */
int des_shade_forward(const des_shade_args* args, unsigned flags, float* shading, float* diffuse_shading,
                      void* workspace, size_t workspace_bytes, des_stream_t stream);

/* Adjoint of des_shade_forward.  grad_diffuse_shading may be NULL (treated as zero).  Outputs
 * g_view_dir, g_albedo, g_specular_albedo, g_roughness may be NULL when not wanted; terms that are
 * switched off produce zeros.  g_envmap[C x H x W] is overwritten (not accumulated); its cross-block
 * sum runs in FP64 on the device and is deterministic.
 * Replaces the kernel pairs behind the reference's *_backward / *_backward2 entry points
 * (bruteforce_shader.cu:2735-2792, 2846-2949, 3002-3106, 3167-3259, 3338-3453). */
int des_shade_backward(const des_shade_args* args, unsigned flags, const float* grad_shading,
                       const float* grad_diffuse_shading, float* g_normal, float* g_view_dir, float* g_albedo,
                       float* g_specular_albedo, float* g_roughness, float* g_envmap, void* workspace,
                       size_t workspace_bytes, des_stream_t stream);

/* Size of the static device scratch array used by des_shade_backward_noalloc. */
#define DES_SHADE_NOALLOC_SCRATCH_BYTES (4u << 20)

/* des_shade_backward for callers that cannot allocate device memory (no counterpart in the
 * reference).  Same inputs and outputs as des_shade_backward, no workspace argument: scratch comes
 * from a library-owned static device array of DES_SHADE_NOALLOC_SCRATCH_BYTES, held on every GPU
 * that uses it until the process exits.  Returns DES_ERR_WORKSPACE, without launching anything,
 * when des_shade_workspace_bytes(P, H, W, flags | DES_COMPACT, 1, device) exceeds that size
 * (a problem that fits only a smaller plan runs with that plan, see DES_COMPACT).  All calls share the
 * array: calls whose work overlaps on the GPU race and corrupt each other.  The first call on each
 * device looks up the array's address (cudaGetSymbolAddress); make it before any stream capture.
 * DES_REUSE_ORDER and DES_REUSE_TABLE are ignored (the array never holds a forward's state).  Out-of-range mesh ids
 * found on the device shade to zero but are not reported (there is no caller-visible workspace for
 * des_workspace_status to read).  Allocates nothing. */
int des_shade_backward_noalloc(const des_shade_args* args, unsigned flags, const float* grad_shading,
                               const float* grad_diffuse_shading, float* g_normal, float* g_view_dir,
                               float* g_albedo, float* g_specular_albedo, float* g_roughness, float* g_envmap,
                               des_stream_t stream);

/* ---------------------------------------------------------------------------------------
 * Multi-env-map relighting (tensor cores)
 * ------------------------------------------------------------------------------------- */

/* Scratch bytes of des_relight_multienv for P points, an H x W map and K env maps. */
size_t des_relight_workspace_bytes(int64_t P, int32_t H, int32_t W, int32_t K);

/* out[P x K x 3] = the forward shading of the P points under each of K env maps
 * (envmaps: K x 3 x H x W float32; args->envmap is ignored), i.e. K calls of the reference's
 * bruteforce_specularvisibility_shader_forward2 (bruteforce_shader.cu:3261) -- or of
 * bruteforce_specular_shader_forward2 without visibility -- fused into one pass whose
 * point x texel weights are contracted with the K maps on tcgen05 (BF16 in, FP32 accumulate).
 * flags: DES_DIFFUSE | DES_SPECULAR [| DES_CLAMP] [| DES_RELIGHT_BF16].  H*W <= 2048. */
int des_relight_multienv(const des_shade_args* args, const float* envmaps, int32_t K, unsigned flags, float* out,
                         void* workspace, size_t workspace_bytes, des_stream_t stream);

/* ---------------------------------------------------------------------------------------
 * Serving: continuous batching of shading requests (no reference counterpart; the reference
 * is a per-call library, bruteforce_shader.cu:3261-3453 is its per-request path)
 * ------------------------------------------------------------------------------------- */

typedef struct des_server des_server;

/* One request.  All pointers are host memory, pinned (cudaMallocHost / torch pin_memory) for
 * asynchronous copies, and must stay valid until the request is reported done. */
typedef struct des_serve_request {
  int64_t P;
  int32_t env_id;   /* from des_server_add_envmap */
  int32_t mesh_id;  /* from des_server_add_mesh, or -1 for no visibility */
  unsigned flags;   /* DES_DIFFUSE | DES_SPECULAR [| DES_CLAMP] */
  int32_t backward; /* 0: shading only; 1: shading and all gradients */
  const float* normal;
  const float* view_dir;
  const float* albedo;
  const float* specular_albedo;
  const float* roughness;
  const int64_t* nearest_triangle_id; /* P, when mesh_id >= 0 */
  const float* barycentric_coord;     /* 3 x P, when mesh_id >= 0 */
  const float* grad_shading;          /* P x 3, when backward */
  const float* grad_diffuse_shading;  /* P x 3 or NULL, when backward */
  float* shading;                     /* P x 3 out */
  float* diffuse_shading;             /* P x 3 out, or NULL */
  float* g_normal;                    /* backward outputs (each may be NULL) */
  float* g_view_dir;
  float* g_albedo;
  float* g_specular_albedo;
  float* g_roughness;
  float* g_envmap; /* 3 x H x W */
} des_serve_request;

typedef struct des_serve_done {
  int64_t ticket;
  /* steady clock, relative to server creation: submitted, admitted (memory reserved), inputs on
   * the device, points ordered (ready to shade), last tile computed, outputs in host memory */
  int64_t t_submit_ns, t_admit_ns, t_uploaded_ns, t_ready_ns, t_computed_ns, t_done_ns;
  int32_t status;
  int32_t pad;
} des_serve_done;

typedef struct des_serve_stats {
  int64_t submitted, completed, ticks, items, peak_arena_bytes;
  int32_t device_error; /* error word of the batch kernel: 1 bad mesh index, 4 malformed work item,
                           8 bad permutation entry; 16 marks a tick that ran without its graph */
  int32_t pad;
} des_serve_stats;

/* Starts a server on `device` with a device arena of hbm_budget_bytes (requests are admitted only
 * while their buffers fit) and a scheduling tick of about tick_us microseconds of GPU work. */
int des_server_create(int device, size_t hbm_budget_bytes, int tick_us, des_server** out);
/* Registers a resident env map (3 x H x W radiance and 3 x 3 rotation, host or device memory). */
int des_server_add_envmap(des_server* s, int32_t H, int32_t W, const float* envmap, const float* light2obj_rotmat,
                          int32_t* env_id);
/* Registers a resident mesh: faces (3 x N_face) and visibility words (N_slot x N_vertex). */
int des_server_add_mesh(des_server* s, int32_t N_face, int32_t N_vertex, int32_t N_slot,
                        const int32_t* face_vertex_list, const int32_t* visibility, int32_t* mesh_id);
/* Queues a request; returns immediately with its ticket (DES_ERR_INVALID_ARGUMENT, and no ticket,
 * for a malformed request).  A request whose buffers could never fit the HBM budget finishes at
 * once with status DES_ERR_WORKSPACE.  After a CUDA error the server fails every outstanding
 * request (status DES_ERR_CUDA in des_serve_done) and refuses new ones.  When every
 * output the request names is device memory of the server's device, or pinned host memory and the
 * request is shaded in input order, the batch kernel stores the results there directly; otherwise
 * they are staged in the arena and copied back.  Either way they are in place when the request is
 * reported done.  A request shaded in input order whose inputs are all device memory of the
 * server's device or pinned host memory is read in place (no upload); other requests' inputs are
 * copied into the arena.  The caller keeps every buffer valid and unchanged until the request is
 * reported done. */
int des_server_submit(des_server* s, const des_serve_request* req, int64_t* ticket);
/* Moves up to max_items finished requests (outputs already in the caller's memory) into out[]. */
int des_server_poll(des_server* s, des_serve_done* out, int max_items, int* count);
/* Waits until every submitted request has finished (DES_ERR_TIMEOUT after timeout_ms). */
int des_server_drain(des_server* s, int timeout_ms);
/* How many ticks may be queued on the GPU at once (1..4, default 4): more overlaps consecutive
 * ticks better, fewer lets a newly arrived request start sooner. */
int des_server_set_ticks_in_flight(des_server* s, int n);
/* Requests of at least n points (and at least 16384) are ordered by normal direction before they
 * are shaded; smaller ones are shaded in input order (by default no request is ordered).  Applies
 * to requests admitted after the call. */
int des_server_set_order_min_points(des_server* s, int64_t n);
/* Scheduling order of the ready requests (and of their uploads): least remaining points x texels
 * first (enable = 1, the default), which ranks a request that asks for gradients like the same
 * request without them, or least remaining work first (enable = 0; an adjoint pair counts twice).
 * Applies to requests admitted after the call. */
int des_server_set_rank_by_size(des_server* s, int enable);
int des_server_stats(des_server* s, des_serve_stats* out);
/* Finishes queued work and frees the server. */
int des_server_destroy(des_server* s);

/* ---------------------------------------------------------------------------------------
 * Mesh-side helpers of the visibility path (reference etc.cu)
 * ------------------------------------------------------------------------------------- */

/* barycentric_coord[P x 3] = (1 - s - t, s, t) of the point of triangle p closest to query_pos[p];
 * triangles: P x 3 vertices x 3 floats.  Replaces get_uv_of_triangle_forward (etc.cu:1218). */
int des_get_uv_of_triangle_forward(int64_t P, const float* triangles, const float* query_pos,
                                   float* barycentric_coord, des_stream_t stream);
/* grad_query_pos[P x 3] from grad_barycentric_coord[P x 3].  Replaces get_uv_of_triangle_backward
 * (etc.cu:1246). */
int des_get_uv_of_triangle_backward(int64_t P, const float* triangles, const float* query_pos,
                                    const float* grad_barycentric_coord, float* grad_query_pos, des_stream_t stream);
/* Nearest point of the mesh to each query among the faces adjacent to its K nearest vertices
 * (idxs[P x K], int64; negative entries are skipped).  adjacency_head[2 x N_vertex] holds per vertex
 * its face count and the inclusive prefix sum of the counts into adjacency_list[N_adj].  Outputs
 * nearest_triangle_id[P] (int64) and barycentric_coord[3 x P]; a query with no candidate face gets
 * id -1 and zero coordinates and sets bit 0 of *error_word (optional, device memory).  Out-of-range
 * ids in the inputs are skipped.  Replaces get_nearest_mesh_points_forward (etc.cu:1277). */
int des_get_nearest_mesh_points_forward(int32_t N_vertex, int32_t N_face, int64_t P, int32_t K, int64_t N_adj,
                                        const int32_t* adjacency_head, const int32_t* adjacency_list,
                                        const int32_t* face_vertex_list, const float* vertex_pos,
                                        const float* query_pos, const int64_t* idxs, int64_t* nearest_triangle_id,
                                        float* barycentric_coord, unsigned* error_word, des_stream_t stream);
/* grad_query_pos[3 x P] from grad_barycentric_coord[3 x P] through the closest-point map of each
 * query's nearest triangle.  Replaces get_nearest_mesh_points_backward (etc.cu:1328), using the
 * incoming gradient where the reference kernel reads its uninitialised output (etc.cu:884-888). */
int des_get_nearest_mesh_points_backward(int32_t N_vertex, int32_t N_face, int64_t P, const int32_t* face_vertex_list,
                                         const float* vertex_pos, const float* query_pos,
                                         const int64_t* nearest_triangle_id, const float* grad_barycentric_coord,
                                         float* grad_query_pos, unsigned* error_word, des_stream_t stream);
/* out[(i_end - i_start) x N_bit] = bit k of the visibility words of point i (1.0f / 0.0f), from
 * bitfield[N_slot x N] (texel k at bit k % 32 of slot k / 32).  Replaces extract_bitfield_forward
 * (etc.cu:1044). */
int des_extract_bitfield_forward(int32_t N_slot, int32_t N, int32_t N_bit, int32_t i_start, int32_t i_end,
                                 const int32_t* bitfield, float* out, des_stream_t stream);

/* ---------------------------------------------------------------------------------------
 * Env-map preprocessing (reference etc.cu)
 * ------------------------------------------------------------------------------------- */

/* out[C x P] = bilinear lat-long lookup of envmap[C x H x W] in the directions query_point[3 x P]
 * (normalised here; columns wrap at the seam, rows clamp at the poles).  Replaces
 * sample_envmap_forward (etc.cu:1145), which allocates 3 x P whatever C is. */
int des_sample_envmap_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* query_point,
                              const float* envmap, float* out, des_stream_t stream);
/* out[C x tar_H x tar_W] = per output texel the mean of N_samples lookups of envmap[C x H x W] in
 * directions drawn from the GGX distribution of roughness parameter alpha around the texel's
 * direction (curand XORWOW, seed 0, one subsequence per texel, as the reference).  C is 3 or 4.
 * Replaces blur_envmap_forward (etc.cu:1103). */
int des_blur_envmap_forward(int32_t H, int32_t W, int32_t C, int32_t tar_H, int32_t tar_W, int32_t N_samples,
                            float alpha, const float* envmap, float* out, des_stream_t stream);

/* The rotated texel table the kernels integrate over, written to table_out[H*W x 4] as
 * (x, y, z, d_omega) per texel in memory order.  Bit-exact with the reference's per-pair
 * getLightDir / getDeltaOmega / rotation (bruteforce_shader.cu:124-147, 2174-2197). */
int des_texel_table(int32_t H, int32_t W, const float* light2obj_rotmat, float* table_out, des_stream_t stream);

/* Instrumentation.  While both events are set (non-NULL cudaEvent_t handles), every shading call
 * records `start_event` on its stream immediately before its main kernel (the forward sum, the
 * fused adjoint, or the first tensor-core pass of des_relight_multienv) and `stop_event`
 * immediately after it, so the caller can time that kernel alone.
 * Process-wide; pass NULL, NULL to turn it off. */
int des_set_timing_events(void* start_event, void* stop_event);

/* Number of kernels this library has launched since it was loaded, on every stream and device
 * (a served tick counts once, whether it ran as a CUDA graph or as a plain launch).  Read it
 * before and after a region to count the launches inside it. */
unsigned long long des_kernel_launches(void);

/* Copies the device-side error word of a workspace used by a finished call to *status_out
 * (DES_OK or DES_ERR_BAD_INDEX) and clears it.  Synchronises `stream`. */
int des_workspace_status(void* workspace, size_t workspace_bytes, int* status_out, des_stream_t stream);

/* ---------------------------------------------------------------------------------------
 * Reference-named entry points: the reference's argument order with tensors as pointers.
 * Each one replaces the pybind function of the same name (bindings.cpp:6-19).
 * ------------------------------------------------------------------------------------- */

/* bruteforce_shader.cu:2687 / gsface_shader.h:1 */
int des_bruteforce_diffuse_shader_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                          const float* albedo, const float* envmap, const float* light2obj_rotmat,
                                          float* shading, void* workspace, size_t workspace_bytes,
                                          des_stream_t stream);
/* bruteforce_shader.cu:2735 / gsface_shader.h:8 */
int des_bruteforce_diffuse_shader_backward(int64_t P, int32_t H, int32_t W, int32_t C, const float* grad_shading,
                                           const float* normal, const float* albedo, const float* envmap,
                                           const float* light2obj_rotmat, float* grad_normal, float* grad_albedo,
                                           float* grad_envmap, void* workspace, size_t workspace_bytes,
                                           des_stream_t stream);
/* bruteforce_shader.cu:2796 (clamp = 0) and 2953 (clamp = 1) / gsface_shader.h:16, 40 */
int des_bruteforce_specular_shader_forward(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                           const float* view_dir, const float* albedo,
                                           const float* specular_albedo, const float* roughness,
                                           const float* envmap, const float* light2obj_rotmat, int enable_diffuse,
                                           int enable_specular, int clamp, float* shading, void* workspace,
                                           size_t workspace_bytes, des_stream_t stream);
/* bruteforce_shader.cu:2846 (clamp = 0) and 3002 (clamp = 1) / gsface_shader.h:27, 51 */
int des_bruteforce_specular_shader_backward(int64_t P, int32_t H, int32_t W, int32_t C, const float* grad_shading,
                                            const float* normal, const float* view_dir, const float* albedo,
                                            const float* specular_albedo, const float* roughness,
                                            const float* envmap, const float* light2obj_rotmat,
                                            int enable_diffuse, int enable_specular, int clamp,
                                            float* grad_normal, float* grad_view_dir, float* grad_albedo,
                                            float* grad_specular_albedo, float* grad_roughness,
                                            float* grad_envmap, void* workspace, size_t workspace_bytes,
                                            des_stream_t stream);
/* bruteforce_shader.cu:3108 / gsface_shader.h:64 */
int des_bruteforce_specular_shader_forward2(int64_t P, int32_t H, int32_t W, int32_t C, const float* normal,
                                            const float* view_dir, const float* albedo,
                                            const float* specular_albedo, const float* roughness,
                                            const float* envmap, const float* light2obj_rotmat,
                                            int enable_specular, float* shading, float* diffuse_shading,
                                            void* workspace, size_t workspace_bytes, des_stream_t stream);
/* bruteforce_shader.cu:3167 / gsface_shader.h:75 */
int des_bruteforce_specular_shader_backward2(int64_t P, int32_t H, int32_t W, int32_t C,
                                             const float* grad_shading, const float* grad_diffuse_shading,
                                             const float* normal, const float* view_dir, const float* albedo,
                                             const float* specular_albedo, const float* roughness,
                                             const float* envmap, const float* light2obj_rotmat,
                                             int enable_specular, float* grad_normal, float* grad_view_dir,
                                             float* grad_albedo, float* grad_specular_albedo,
                                             float* grad_roughness, float* grad_envmap, void* workspace,
                                             size_t workspace_bytes, des_stream_t stream);
/* bruteforce_shader.cu:3261 / gsface_shader.h:88 */
int des_bruteforce_specularvisibility_shader_forward2(
    int64_t P, int32_t H, int32_t W, int32_t C, int32_t N_face, int32_t N_vertex, int32_t N_slot,
    const float* normal, const float* view_dir, const float* albedo, const float* specular_albedo,
    const float* roughness, const float* envmap, const float* light2obj_rotmat, const int32_t* face_vertex_list,
    const int64_t* nearest_triangle_id, const float* barycentric_coord, const int32_t* visibility,
    int enable_specular, float* shading, float* diffuse_shading, void* workspace, size_t workspace_bytes,
    des_stream_t stream);
/* bruteforce_shader.cu:3338 / gsface_shader.h:103 */
int des_bruteforce_specularvisibility_shader_backward2(
    int64_t P, int32_t H, int32_t W, int32_t C, int32_t N_face, int32_t N_vertex, int32_t N_slot,
    const float* grad_shading, const float* grad_diffuse_shading, const float* normal, const float* view_dir,
    const float* albedo, const float* specular_albedo, const float* roughness, const float* envmap,
    const float* light2obj_rotmat, const int32_t* face_vertex_list, const int64_t* nearest_triangle_id,
    const float* barycentric_coord, const int32_t* visibility, int enable_specular, float* grad_normal,
    float* grad_view_dir, float* grad_albedo, float* grad_specular_albedo, float* grad_roughness,
    float* grad_envmap, void* workspace, size_t workspace_bytes, des_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DIFF_ENVSHADE_B200_H_ */
