/*
 * rtrace_gpu.h -- C ABI of the B200 render path for SeaRyanC/rtrace scenes.
 *
 * The reference renders through the Rust API `Renderer::render(&self,
 * &Scene) -> Result<RgbImage, Box<dyn Error>>` (src/renderer.rs:120) and
 * `Renderer::render_to_file` (src/renderer.rs:914).  This header is what a
 * Rust (or any C-FFI) host binds to replace that body: scenes are loaded
 * once into a device-resident handle, and each render call takes the
 * `Renderer` fields (src/renderer.rs:37-47) and fills a caller-owned RGB8
 * buffer with the bytes `create_image_from_data` (src/renderer.rs:899-912)
 * would produce.
 *
 * Conventions
 *   - Every entry point returns an rt_status; nothing throws across the ABI.
 *     The message of the last failure on a context is rt_last_error(ctx).
 *   - Caller buffers are borrowed for the duration of the call; device
 *     memory belongs to the context (or to the scene handle).
 *   - A context owns one CUDA stream.  Calls on one context must not
 *     overlap; use one context per host thread for concurrency (render
 *     calls are re-entrant in the reference: src/renderer.rs:120 takes
 *     &self and builds its world per call).
 */
#ifndef RTRACE_GPU_H
#define RTRACE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports errors as strings inside a
 * Result; RT_ERR_SCENE covers Scene::from_json_file/from_json_str failures
 * (src/scene.rs:462-505, src/mesh.rs:751-1003) and RT_ERR_RENDER covers the
 * errors Renderer::render returns: "Samples must be greater than 0"
 * (src/renderer.rs:122-124), "Field of view must be between 0 and 180
 * degrees" (src/camera.rs:115-117), "Unsupported camera type: ..."
 * (src/camera.rs:62), "Invalid hex color..." (src/scene.rs:15-30) and the
 * panics of rand's gen_range on an empty range (a disk light of zero or
 * negative diameter).  The remaining codes are GPU-side failures the
 * reference cannot have. */
typedef enum rt_status {
  RT_OK = 0,
  RT_ERR_INVALID_ARGUMENT = 1,
  RT_ERR_SCENE = 2,
  RT_ERR_RENDER = 3,
  RT_ERR_CUDA = 4,
  RT_ERR_OUT_OF_MEMORY = 5,
  RT_ERR_DEVICE_WATCHDOG = 6, /* a bounded device loop ran out of iterations */
  RT_ERR_IO = 7
} rt_status;

/* AntiAliasingMode (src/renderer.rs:16-24). */
typedef enum rt_aa_mode {
  RT_AA_NO_JITTER = 0,
  RT_AA_QUINCUNX = 1,
  RT_AA_STOCHASTIC = 2
} rt_aa_mode;

typedef struct rt_ctx rt_ctx;     /* device, stream and scratch buffers */
typedef struct rt_scene rt_scene; /* device-resident flattened world */

/* OutlineConfig (src/outline.rs:5-31).  Applied only in the no-jitter and
 * stochastic modes, as src/renderer.rs:409-410 ignores it in quincunx. */
typedef struct rt_outline_config {
  int32_t enabled;
  int32_t use_8_neighbors;
  double depth_weight;
  double normal_weight;
  double threshold;
  double edge_color[3];
  double line_thickness;
  /* Extension (0 keeps the reference's outline): weight of an edge term
   * between neighbouring foreground pixels whose nearest samples hit
   * different World objects, added to the depth and normal terms.  Renders
   * take the objects from their own hit records; rt_outline_apply has no
   * object buffer and ignores it. */
  double object_id_weight;
} rt_outline_config;

/* Renderer fields (src/renderer.rs:37-47).  thread_count has no device
 * meaning and is not carried.  seed: `None` is rendered as 0, exactly as
 * `self.seed.unwrap_or(0)` does.  flags: RT_FLAG_* (profiling, graph replay). */
typedef struct rt_render_params {
  uint32_t width;
  uint32_t height;
  int32_t max_depth;
  int32_t use_kdtree;
  uint32_t samples;
  int32_t anti_aliasing_mode; /* rt_aa_mode */
  uint64_t seed;
  rt_outline_config outline;
  uint32_t flags;
  uint32_t reserved;
  /* Extensions with no counterpart in the reference; zero keeps its
   * behaviour.  disk_samples: shadow rays per disk light and shading point
   * (0 means 16, the reference's constant; more samples continue the same
   * StdRng stream).  learned_shadows: primary hits cast one ray per disk
   * light and the learned denoiser (rt_denoiser_load) estimates each disk
   * light's visibility from those rays and the hit's G-buffer; the light
   * then contributes its light-centre term times the squared estimate. */
  uint32_t disk_samples;
  int32_t learned_shadows;
  /* learned_shadows: rays per disk light at the primary hits (1..16); 0
   * uses the count the loaded network was trained on. */
  uint32_t learned_rays;
  /* learned_shadows with a network that estimates its own error (blob
   * version 3): a primary hit's disk light whose estimated visibility error
   * exceeds confidence_threshold is shaded by the plain path instead, with
   * fallback_samples rays (0: as disk_samples), the first samples of the
   * reference's StdRng stream.
   * confidence_threshold 0 uses the threshold stored with the weights; a
   * negative value turns the fallback off. */
  uint32_t fallback_samples;
  float confidence_threshold;
  uint32_t reserved3;
} rt_render_params;

/* Profiling flags: per-stage CUDA-event times, and device work counters
 * (node visits, primitive tests).  Both slow the render slightly. */
#define RT_FLAG_STAGE_TIMES 1u
#define RT_FLAG_COUNT_WORK 2u
/* Launch the frame as a CUDA graph.  The first render with a given set of
 * launch arguments (scene, camera, image size, parameters, output pointer)
 * captures its kernel sequence; later identical renders replay it in one
 * submission.  Ignored with RT_FLAG_STAGE_TIMES and by rt_render_linear.
 * The image is the same either way. */
#define RT_FLAG_CUDA_GRAPH 4u

/* Stages reported in rt_stats.stage_ms */
enum { RT_STAGE_RAYGEN = 0, RT_STAGE_TRACE = 1, RT_STAGE_EMIT = 2, RT_STAGE_SHADOW = 3, RT_STAGE_RESOLVE = 4,
       RT_STAGE_FOLD = 5, RT_STAGE_POST = 6, RT_STAGE_DENOISE = 7, RT_STAGE_COUNT = 8 };

/* Counters of one render.  Rays are counted the way the reference casts
 * them: primary (one per camera sample; quincunx casts W*H centre rays and
 * (W+1)*(H+1) corner rays), reflection (one per recursive ray_color call)
 * and shadow (one per World::hit issued by a light). */
typedef struct rt_stats {
  uint64_t primary_rays;
  uint64_t reflection_rays;
  uint64_t shadow_rays;
  uint64_t hits;            /* closest-hit queries that hit an object */
  /* RT_FLAG_COUNT_WORK: work of the closest-hit (trace) and shadow (any-hit)
   * kernels: acceleration nodes visited, triangle and sphere tests, and
   * reference-leaf verifications of mesh candidates */
  uint64_t trace_nodes, trace_triangles, trace_spheres, trace_verifications;
  uint64_t shadow_nodes, shadow_triangles, shadow_spheres, shadow_verifications;
  uint32_t kernel_launches; /* kernels this render launched */
  uint32_t graph;           /* RT_FLAG_CUDA_GRAPH: 1 captured by this call, 2 replayed; 0 launched directly */
  double device_ms; /* CUDA-event time of the device pipeline */
  double total_ms;  /* host wall time of the whole call */
  double stage_ms[RT_STAGE_COUNT]; /* RT_FLAG_STAGE_TIMES */
  uint64_t fallback_hits;   /* learned shadows: primary hits with a light shaded by the plain fallback */
  uint64_t fallback_lights; /* learned shadows: (primary hit, disk light) pairs shaded by the fallback */
  /* Shadow rays (counted in shadow_rays, which counts the rays the
   * reference casts) that were not traced because the surface faces away
   * from the light: the reference's contribution of that light is exactly
   * zero whatever they hit. */
  uint64_t shadow_rays_untraced;
} rt_stats;

/* ------------------------------------------------------------------ */
/* Flattened scene description, for hosts that build their own world   */
/* (the reference's World build, src/renderer.rs:138-317, done by the  */
/* caller).  All pointers are borrowed during rt_scene_upload only.     */
/* ------------------------------------------------------------------ */

/* scene::Camera (src/scene.rs:33-46).  kind is the JSON string. */
typedef struct rt_camera_config {
  char kind[32];
  double position[3];
  double target[3];
  double up[3];
  double width;
  double height;
  int32_t has_fov;
  int32_t has_grid_pitch;
  int32_t has_grid_thickness;
  int32_t grid_color_state; /* 0 absent, 1 parsed, 2 unparsable (render error) */
  double fov;
  double grid_pitch;
  double grid_thickness;
  double grid_color[3];
} rt_camera_config;

/* scene::Material (src/scene.rs:66-89) with its colours already parsed the
 * way phong_lighting/apply_texture parse them (src/lighting.rs:9-54,
 * 229-248). */
typedef struct rt_material_desc {
  double color[3];
  double ambient, diffuse, specular, shininess;
  int32_t has_reflectivity;
  int32_t texture; /* 0 none, 1 grid, 2 checkerboard */
  double reflectivity;
  double grid_line_color[3]; /* hex_to_color(line_color).unwrap_or(black) */
  double grid_line_width;
  double grid_cell_size;
  double checker_color[3]; /* material_b colour, unwrap_or(white) */
  double checker_ambient, checker_diffuse, checker_specular, checker_shininess;
} rt_material_desc;

typedef enum rt_object_kind {
  RT_OBJ_SPHERE = 0,
  RT_OBJ_PLANE = 1,
  RT_OBJ_CUBE = 2,
  RT_OBJ_MESH = 3
} rt_object_kind;

/* One World entry in scene order (src/ray.rs:683-712), primitives already
 * transformed as src/renderer.rs:141-310 does. */
typedef struct rt_object_desc {
  int32_t kind;          /* rt_object_kind */
  int32_t material;      /* material index (the object's scene index) */
  double a[3];           /* sphere/cube centre, plane point */
  double b[3];           /* plane normal (normalised), cube size */
  double radius;         /* sphere radius (after max column scale) */
  int32_t has_transform; /* cube: transform[] holds its matrix */
  int32_t mesh;          /* mesh: index into rt_scene_desc.meshes */
  double transform[16];  /* cube local-to-world matrix, row-major */
} rt_object_desc;

/* KdNode (src/mesh.rs:41-55) in preorder; the left child of an internal
 * node is the next node. */
typedef struct rt_kd_node_desc {
  int32_t axis;  /* 0..2 internal node, -1 leaf */
  int32_t right; /* internal: index of the right child */
  int32_t first; /* leaf: first entry in tri_index */
  int32_t count; /* leaf: number of entries */
  double split;
  double bounds_min[3];
  double bounds_max[3];
} rt_kd_node_desc;

/* Mesh (src/mesh.rs:730-1050) after its transform, with its k-d tree. */
typedef struct rt_mesh_desc {
  const double* vertices; /* 9 doubles per triangle: v0, v1, v2 */
  int64_t n_triangles;
  double bounds_min[3];
  double bounds_max[3];
  const rt_kd_node_desc* nodes; /* may be NULL when the mesh is empty */
  int64_t n_nodes;
  const int32_t* tri_index; /* leaf triangle lists, leaf order */
  int64_t n_tri_index;
} rt_mesh_desc;

/* scene::Light (src/scene.rs:347-353), colour parsed unwrap_or(white). */
typedef struct rt_light_desc {
  double position[3];
  double color[3];
  double intensity;
  int32_t has_diameter;
  int32_t pad;
  double diameter;
} rt_light_desc;

typedef struct rt_scene_desc {
  rt_camera_config camera;
  const rt_object_desc* objects;
  int32_t n_objects;
  int32_t n_materials;
  const rt_material_desc* materials;
  const rt_light_desc* lights;
  int32_t n_lights;
  int32_t n_meshes;
  const rt_mesh_desc* meshes;
  double ambient_color[3]; /* unwrap_or(white) */
  double ambient_intensity;
  int32_t has_fog;
  int32_t has_outline; /* scene_settings.outline present and enabled */
  double fog_color[3]; /* unwrap_or(0.5 grey) */
  double fog_density, fog_start, fog_end;
  double background[3];
  rt_outline_config outline; /* Scene::get_outline_config (src/scene.rs:515-534) */
  /* First error Renderer::render would raise while building its world
   * (an unparsable material or background colour), or NULL. */
  const char* render_error;
} rt_scene_desc;

/* ------------------------------------------------------------------ */
/* Entry points                                                         */
/* ------------------------------------------------------------------ */

/* Creates a context on CUDA device `device`. */
rt_status rt_ctx_create(int device, rt_ctx** out);
void rt_ctx_destroy(rt_ctx* ctx);
/* Message of the last failure on ctx ("" if none).  Valid until the next
 * call on ctx.  rt_last_error(NULL) reports failures of rt_ctx_create. */
const char* rt_last_error(const rt_ctx* ctx);

/* Scene::from_json_file (src/scene.rs:462-470): parse, load STL meshes
 * relative to the file's directory, transform, build k-d trees, upload. */
rt_status rt_scene_load_json_file(rt_ctx* ctx, const char* path, rt_scene** out);
/* Scene::from_json_str (src/scene.rs:473-480): meshes relative to ".". */
rt_status rt_scene_load_json_str(rt_ctx* ctx, const char* json, rt_scene** out);
/* Uploads a world the caller flattened itself. */
rt_status rt_scene_upload(rt_ctx* ctx, const rt_scene_desc* desc, rt_scene** out);
/* Scene::get_outline_config (src/scene.rs:515-534) of a loaded scene;
 * *enabled = 0 when the scene has none. */
rt_status rt_scene_outline_config(rt_ctx* ctx, const rt_scene* scene, rt_outline_config* out);
/* Camera aspect (camera.width / camera.height) used by the CLI and the
 * Node bindings to size images from a diagonal (cli/src/main.rs:339-350). */
rt_status rt_scene_camera_aspect(rt_ctx* ctx, const rt_scene* scene, double* out);
void rt_scene_free(rt_scene* scene);

/* Host-side scene: Scene::from_json_file / from_json_str parsed, meshes
 * loaded and transformed and k-d trees built, with nothing on the device
 * yet.  rt_host_scene_desc exposes the flattened description that
 * rt_scene_upload takes (valid until rt_host_scene_free).  Errors are
 * reported through rt_last_error(NULL). */
typedef struct rt_host_scene rt_host_scene;
rt_status rt_host_scene_load_json_file(const char* path, rt_host_scene** out);

/* AutoCamera::generate_cameras (src/auto_camera.rs:9-130) over
 * Scene::compute_finite_bounds (src/scene.rs:538-690): writes the left,
 * front, top and perspective cameras, in that order, to out[0..3].  Fails
 * with the scene's parse error or "Scene has no finite objects to compute
 * bounds" (reported by rt_last_error(NULL)). */
rt_status rt_auto_cameras_json_file(const char* path, rt_camera_config* out);
rt_status rt_auto_cameras_json_str(const char* json, rt_camera_config* out);
rt_status rt_host_scene_load_json_str(const char* json, rt_host_scene** out);
/* The same loads with the k-d trees of meshes of 16,384 triangles or more
 * built on ctx's device (rt_kd_build); the host scene is identical.
 * rt_scene_load_json_file / _str build the same way.  Errors are reported
 * through rt_last_error(ctx). */
rt_status rt_host_scene_load_json_file_on(rt_ctx* ctx, const char* path, rt_host_scene** out);
rt_status rt_host_scene_load_json_str_on(rt_ctx* ctx, const char* json, rt_host_scene** out);
const rt_scene_desc* rt_host_scene_desc(const rt_host_scene* hs);
void rt_host_scene_free(rt_host_scene* hs);

/* rt_scene_upload of a host scene's own description.  The first upload
 * prepares the meshes' device data on the host (BVH, triangle records,
 * k-d root paths and occurrence lists) and keeps it in the host scene;
 * later uploads of the same host scene, to any context, only copy it. */
rt_status rt_host_scene_upload(rt_ctx* ctx, rt_host_scene* hs, rt_scene** out);
/* KdTree::new(triangles, 16, 10) (src/mesh.rs:75-197, the tree
 * Mesh::from_stl_file and the World build make) over n_triangles of 9
 * doubles each (v0, v1, v2), as rt_mesh_desc wants it: nodes in preorder
 * and the leaf lists.  With a context it is built on that device, one tree
 * depth at a time; with ctx NULL on the host.  Both give the same bytes.
 * A NaN centre in a node the reference sorts fails with RT_ERR_SCENE and
 * the reference's panic message (its sort unwraps partial_cmp). */
typedef struct rt_kd_tree rt_kd_tree;
rt_status rt_kd_build(rt_ctx* ctx, const double* vertices, int64_t n_triangles, rt_kd_tree** out);
const rt_kd_node_desc* rt_kd_tree_nodes(const rt_kd_tree* tree, int64_t* n_nodes);
const int32_t* rt_kd_tree_index(const rt_kd_tree* tree, int64_t* n_index);
void rt_kd_tree_free(rt_kd_tree* tree);

/* PNG output (Renderer::render_to_file, src/renderer.rs:914-920): an
 * 8-bit RGB image (width*height*3 bytes, top row first) as a PNG, encoded
 * on the host's threads (adaptive row filters, the deflate stream cut into
 * bands compressed in parallel).  The decoded pixels are the image; the
 * file bytes differ from the reference's encoder.  rt_png_encode returns a
 * buffer to release with rt_png_free; level is zlib's 0-9 (-1: default).
 * rt_png_write writes at level 1 and fails with RT_ERR_IO when the file
 * cannot be written. */
rt_status rt_png_encode(const uint8_t* rgb, uint32_t width, uint32_t height, int32_t level, uint8_t** out,
                        size_t* out_len);
void rt_png_free(uint8_t* buffer);
rt_status rt_png_write(const char* path, const uint8_t* rgb, uint32_t width, uint32_t height);

/* Bytes rt_scene_upload copied to the device for this scene. */
rt_status rt_scene_device_bytes(rt_ctx* ctx, const rt_scene* scene, uint64_t* out);

/* Renderer::render (src/renderer.rs:120-382).  rgb_out receives
 * width*height*3 bytes, row-major, top row first.  out_on_device != 0 means
 * rgb_out is a device pointer on the context's device.  stats may be NULL. */
rt_status rt_render(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                    int out_on_device, rt_stats* stats);

/* Rows [row_begin, row_end) of the image rt_render produces, byte for byte
 * (the unit of work of a frame split into row bands across GPUs; the
 * reference renders whole frames only, so there is no single reference
 * function, and the rows are those of Renderer::render, src/renderer.rs:
 * 120-382).  rgb_out receives (row_end - row_begin) * width * 3 bytes.
 * With the outline on, 1 + ceil(thickness - 1) rows beyond each inner band
 * edge are traced as well (the outline stencil reads them); the stats count
 * those rays too. */
rt_status rt_render_rows(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint32_t row_begin,
                         uint32_t row_end, uint8_t* rgb_out, int out_on_device, rt_stats* stats);

/* Same as rt_render but also returns the pre-quantisation colours
 * (width*height*3 doubles, host memory).  Used by parity tests. */
rt_status rt_render_linear(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                           double* linear_out, rt_stats* stats);

/* The outline post-process on its own (apply_outline_detection,
 * src/outline.rs:86-278, then create_image_from_data, src/renderer.rs:
 * 899-912), for hosts that produce their own colour and G-buffers.  All
 * pointers are device memory on the context's device, one value per pixel,
 * row-major: colours r/g/b before quantisation, valid = 1 where the pixel
 * has a depth and normal, depth = camera distance, nx/ny/nz = world normal.
 * rgb_out receives width*height*3 bytes.  config->enabled is ignored. */
rt_status rt_outline_apply(rt_ctx* ctx, uint32_t width, uint32_t height, const double* r, const double* g,
                           const double* b, const uint8_t* valid, const double* depth, const double* nx,
                           const double* ny, const double* nz, const rt_outline_config* config, uint8_t* rgb_out);

/* rt_outline_apply without any device allocation.  No counterpart in the
 * reference (which never touches a GPU); it exists for callers that may
 * not allocate device memory while they run this step: hosts whose device
 * memory is owned by another allocator or arena (an engine or compositor
 * that budgets every byte itself), frame loops where cudaMalloc's implicit
 * device-wide synchronisation would stall their other streams, and
 * long-running services that must not fail with out-of-memory mid-frame.
 *
 * The per-pixel edge-strength scratch lives in one static device array of
 * RT_OUTLINE_NOALLOC_MAX_PIXELS doubles (32 MiB), which every device that
 * loads this library keeps until the process exits; width * height above
 * that limit is rejected with RT_ERR_INVALID_ARGUMENT.  Each call looks up
 * the array's device address on the context's device (cudaGetSymbolAddress;
 * the first lookup on a device also sets up the library's device code
 * there), so make the first call on a device before any stream capture.  All
 * calls share the array: calls whose work overlaps on the GPU (other
 * threads, other contexts on the same device) race on it and must be
 * serialised by the caller.  Nothing in it needs clearing between calls:
 * the mask pass writes every pixel the blend pass reads.  Arguments and
 * results are those of rt_outline_apply. */
#define RT_OUTLINE_NOALLOC_MAX_PIXELS (2048u * 2048u)
rt_status rt_outline_apply_noalloc(rt_ctx* ctx, uint32_t width, uint32_t height, const double* r,
                                   const double* g, const double* b, const uint8_t* valid, const double* depth,
                                   const double* nx, const double* ny, const double* nz,
                                   const rt_outline_config* config, uint8_t* rgb_out);

/* ------------------------------------------------------------------ */
/* Batched rendering (extension: the reference renders one frame per    */
/* Renderer::render call; its CLI's auto-camera mode renders four)      */
/* ------------------------------------------------------------------ */

typedef struct rt_job {
  const rt_scene* scene;          /* uploaded on the batch context's device */
  const rt_camera_config* camera; /* NULL: the scene's camera; else this one (e.g. an auto-camera view) */
  rt_render_params params;
  uint8_t* rgb_out;               /* width * height * 3 bytes, host or device memory */
  int32_t out_on_device;
  int32_t status;                 /* out: this job's rt_status */
  rt_stats stats;                 /* out */
} rt_job;

typedef struct rt_batch_stats {
  uint32_t jobs;
  uint32_t lanes;
  uint64_t rays;          /* primary + reflection + shadow rays of all jobs */
  double wall_ms;         /* host time of the whole batch */
  double device_ms;       /* sum of the jobs' device times */
  double busiest_lane_ms; /* largest per-lane sum of device times */
} rt_batch_stats;

/* Renders n jobs on `lanes` concurrent streams of the context's device
 * (0: the count rt_batch_autotune chose for this context, else 4).  The
 * fused group (rt_batch_tuning.fuse_pixels) goes to lane 0 first; the other
 * jobs are assigned to lanes longest first by their estimated rays (width *
 * height * samples * (1 + shadow rays per hit)) onto the least-loaded lane,
 * so small jobs run beside large ones.  Every job's
 * image is byte for byte the one rt_render gives for the same scene,
 * camera and params.  Returns RT_OK when every job rendered, else the
 * first failing job's status (each job's own status is in jobs[i].status;
 * rt_last_error names the job). */
rt_status rt_render_batch(rt_ctx* ctx, rt_job* jobs, uint32_t n, uint32_t lanes, rt_batch_stats* stats);

/* Launch parameters of rt_render_batch (per context):
 *   lanes: concurrent streams when rt_render_batch gets lanes = 0;
 *   fuse_pixels: frames of at most this many pixels (plain path, no
 *     outline pass, one shadow chunk, no profiling flags) form the fused
 *     group: each wavefront kernel is launched once for all of them over a
 *     device table of their launch blocks, the sequence captured as a CUDA
 *     graph and replayed when the same group comes again (0: no group);
 *   fuse_bytes: the group's frames hold their scratch together, so the
 *     group takes the smallest eligible frames while their estimated
 *     scratch stays within this many bytes (the others render on lanes);
 *   blocks_per_sm: grid budget of each fused kernel kind (ray generation,
 *     closest hit, light sampling, shadow rays, shading, reflection fold,
 *     pixels) in blocks per SM, shared out between the group's frames in
 *     proportion to their work bounds.
 * Defaults: 4 lanes, 640 x 480, 16 GiB, {16, 64, 64, 128, 16, 16, 16}. */
typedef struct rt_batch_tuning {
  uint32_t lanes;
  uint32_t fuse_pixels;
  uint64_t fuse_bytes;
  int32_t blocks_per_sm[7];
  uint32_t trials;  /* out (autotune): batches timed */
  double best_ms;   /* out (autotune): wall time of the chosen parameters */
} rt_batch_tuning;
rt_status rt_batch_get_tuning(rt_ctx* ctx, rt_batch_tuning* out);
rt_status rt_batch_set_tuning(rt_ctx* ctx, const rt_batch_tuning* tuning);

/* Autotuner: renders the batch (twice per candidate: the first run of a new
 * fused group captures its graph) and keeps what is fastest in wall time,
 * one parameter at a time: lanes in {1, 2, 4, 8}; fuse_pixels in {0, 256^2,
 * 640 x 480, 1280 x 720}; then, with a fused group, the blocks per SM of
 * the closest-hit, shadow, light-sampling and shading kernels.  The chosen
 * parameters stay on the context and are returned in *out (may be NULL). */
rt_status rt_batch_autotune_ex(rt_ctx* ctx, rt_job* jobs, uint32_t n, rt_batch_tuning* out);
/* rt_batch_autotune_ex returning only the lane count. */
rt_status rt_batch_autotune(rt_ctx* ctx, rt_job* jobs, uint32_t n, uint32_t* best_lanes);

/* The assignment rt_render_batch makes: job i (estimated cost costs[i])
 * goes to lane lane_of_job[i]; longest job first onto the least-loaded
 * lane, ties to the lower lane. */
rt_status rt_batch_assign(const double* costs, uint32_t n, uint32_t lanes, uint32_t* lane_of_job);

/* ------------------------------------------------------------------ */
/* Learned soft shadows (extension; no counterpart in the reference)  */
/* ------------------------------------------------------------------ */

/* Loads the denoiser's weights into the context (replacing earlier ones).
 * Blob layout, little endian: "RTDN", u32 version, u32 n_ops, then
 *   version 1: per op u32 cin, cout, dilation, activation;
 *   version 2: u32 rays per disk light the network was trained on, then as
 *     version 1;
 *   version 3: u32 rays, f32 default confidence threshold, then per op u32
 *     kind (0 3x3 convolution, 1 2x2 average pooling, 2 nearest 2x
 *     upsampling of buffer src added to buffer src2), cin, cout, dilation,
 *     activation, src, src2 (0xFFFFFFFF: none).
 * Versions 1 and 2 are chains of convolutions (op i reads op i - 1).  In
 * version 3, buffer 0 is the feature image and op i writes buffer i + 1;
 * pooling halves the resolution (rounding up), upsampling joins adjacent
 * resolutions.  Then per convolution FP16 weights [cout][3][3][cin] and
 * FP32 bias [cout].  Convolutions have 16, 32 or 64 input and output
 * channels (16->64 and 64->16 excepted), dilation 1..64 and ReLU
 * (activation 0), except the last op: a full-resolution convolution to 16
 * channels with activation 2 (sigmoid) whose channels 0, 1 are the
 * visibility of disk-light slots 0 and 1 and, in version 3, channels 2, 3
 * the network's estimate of its own absolute error on them. */
rt_status rt_denoiser_load(rt_ctx* ctx, const void* blob, size_t bytes);

/* Runs the loaded denoiser on a feature image ([planes][height][width][16]
 * FP16, device) and writes the visibility estimates ([planes][2][height]
 * [width] float, device) and, if confidence is not NULL and the network has
 * them, its error estimates (same layout).  device_ms (optional): CUDA-event
 * time of the network's kernels. */
rt_status rt_denoiser_run(rt_ctx* ctx, const uint16_t* features, uint32_t planes, uint32_t height, uint32_t width,
                          float* visibility, float* confidence, double* device_ms);

/* ------------------------------------------------------------------ */
/* Denoiser training (extension; no counterpart in the reference)     */
/* ------------------------------------------------------------------ */

/* A trainer holds FP32 master weights, Adam moments and the activations and
 * gradients of one batch shape: planes feature images of height x width.
 * It starts from a version 3 blob (rt_denoiser_load's format).  A step runs
 * the network's forward pass on the inference kernels (masters rounded to
 * FP16), the loss, the backward pass (weight gradients as tcgen05 implicit
 * GEMMs, data gradients as the forward convolution with mirrored,
 * transposed weights) and Adam.  The loss, over the samples whose primary
 * ray hit and whose slot's light exists (features' valid and slot-present
 * channels), is sum (v - t)^2 + (c - |v - t|)^2 with v the visibility
 * output, t the target and c the error output (not differentiated through
 * v).  features: [planes][height][width][16] FP16, targets:
 * [planes][2][height][width] FP16, both device pointers. */
typedef struct rt_dn_trainer rt_dn_trainer;
rt_status rt_dn_train_create(rt_ctx* ctx, const void* blob, size_t bytes, uint32_t planes, uint32_t height,
                             uint32_t width, rt_dn_trainer** out);
/* One optimisation step (Adam with bias correction on the mean loss
 * gradient); loss (optional, host, 4 floats): masked sample count, sum of
 * the visibility term, sum of the error term, and the gradient entries that
 * were not finite (an FP16 activation gradient overflowed; the step is then
 * skipped and the weights keep their values). */
rt_status rt_dn_train_step(rt_dn_trainer* t, const uint16_t* features, const uint16_t* targets, float lr,
                           float beta1, float beta2, float eps, float* loss);
/* The gradient of the summed loss with respect to every parameter (host,
 * FP32, per convolution its weights [cout][3][3][cin] then bias, in op
 * order), without an update; loss as in rt_dn_train_step. */
rt_status rt_dn_train_grads(rt_dn_trainer* t, const uint16_t* features, const uint16_t* targets, float* grads,
                            float* loss);
/* The current weights as a version 3 blob.  blob_out NULL: *bytes receives
 * the size. */
rt_status rt_dn_train_export(rt_dn_trainer* t, void* blob_out, size_t* bytes);
/* The default confidence threshold written by rt_dn_train_export. */
rt_status rt_dn_train_set_threshold(rt_dn_trainer* t, float threshold);
void rt_dn_train_free(rt_dn_trainer* t);
/* Weight and bias gradients of one 3x3 convolution (dilation dil) on the
 * tensor cores: dw[cout][3][3][cin] += sum_q dz[q][co] x[q + tap][ci], db[co]
 * += sum_q dz[q][co]; x [planes][height][width][cin] and dz [..][cout]
 * FP16, dw and db FP32, all device pointers. */
rt_status rt_debug_conv_wgrad(rt_ctx* ctx, const uint16_t* x, const uint16_t* dz, uint32_t planes, uint32_t height,
                              uint32_t width, uint32_t cin, uint32_t cout, uint32_t dil, float* dw, float* db);

/* rt_render plus, for the primary samples (plane = sample index within
 * the pixel, so planes = samples), the shadow visibility each of the first
 * two disk lights got (visible / disk_samples, or the denoised estimate
 * with learned_shadows; meaningful where the feature image says the ray
 * hit) and the denoiser's feature image.  vis and features are device
 * pointers or NULL; rgb_out is host memory or NULL.  No-jitter or
 * stochastic sampling only. */
rt_status rt_render_shadow_aov(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                               float* vis, uint16_t* features, rt_stats* stats);

/* ------------------------------------------------------------------ */
/* Device unit entry points used by the parity tests                   */
/* ------------------------------------------------------------------ */

/* The first n_words u32 outputs of rand's StdRng::seed_from_u64(seed[i])
 * (rand 0.8 / rand_chacha 0.3 ChaCha12, rand_core 0.6 PCG32 seeding) for
 * each of n seeds, generated on the device.  out: n * n_words, host. */
rt_status rt_debug_stdrng_u32(rt_ctx* ctx, const uint64_t* seeds, int64_t n, int32_t n_words, uint32_t* out);
/* The 16 (dx, dy) disk offsets of one area-light shading point
 * (src/lighting.rs:57-66, 170-173) for each light seed; out: n * 32. */
rt_status rt_debug_disk_offsets(rt_ctx* ctx, const uint64_t* light_seeds, int64_t n, double radius, double* out);
/* Measured issue rate of separate FP64 add and multiply instructions (the
 * operations the render path uses; it never fuses them), in Gop/s. */
rt_status rt_debug_fp64_rate(rt_ctx* ctx, double* gops);
/* Measured read bandwidth, in GB/s, of a device buffer of about `bytes`
 * bytes (rounded down to whole passes of the probe's grid; at most 2 GiB)
 * that stays in L2: `reps` passes of 16-byte loads cached in L2 only,
 * after a warm-up pass, timed with CUDA events.  The ceiling of kernels
 * whose working set is L2-resident. */
rt_status rt_debug_l2_read_bandwidth(rt_ctx* ctx, uint64_t bytes, int32_t reps, double* gbs);
/* MeshObject::hit (src/ray.rs:614-675) of mesh `mesh_object` of a loaded
 * scene for n rays (6 doubles each: origin, direction).  out: 8 doubles per
 * ray [hit, t, point xyz, normal xyz].  use_kdtree: bit 0 the Renderer
 * field; bits 1-2 the query: 0 closest hit as rendered, 1 the reference's
 * own k-d walk, 2 any hit below t_max as shadow rays run it, 3 for every
 * k-d leaf the visit test from the leaf's cell against the walk from the
 * root (out: [leaves where they differ, leaves where they agree, leaves
 * the walk visits, 0...]). */
rt_status rt_debug_mesh_hit(rt_ctx* ctx, const rt_scene* scene, int32_t object_index, int32_t use_kdtree,
                            const double* rays, int64_t n, double t_min, double t_max, double* out);
/* Prepares a mesh description's device search data on the host and on
 * the device (the path uploads take for meshes of 262,144 triangles or
 * more; the host preparation of smaller meshes builds its BVH with a
 * binned SAH instead, so the host side here uses the device's median
 * split) and compares them: bit k of *mismatch is set when array k differs
 * (0 BVH, 1 records in BVH order, 2 records in mesh order, 3 normals,
 * 4 k-d occurrences, 5 occurrence offsets).  Bit 6: the arrays that an
 * upload of a host-prepared mesh derives on the device from its BVH-order
 * records and k-d tree (records in mesh order, normals, occurrences) differ
 * from the host's.  Bit 7: the single-precision BVH the walks test (the
 * device's conversion against the host's, which host-prepared uploads
 * copy) differs.  More than 4 triangles (the BVH leaf size). */
rt_status rt_debug_mesh_prep(rt_ctx* ctx, const rt_mesh_desc* mesh, uint32_t* mismatch);

#ifdef __cplusplus
}
#endif

#endif /* RTRACE_GPU_H */
