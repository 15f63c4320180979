// Host-side scene loading: the work the reference does in Rust before its
// render loop (Scene::from_json_file, Mesh::from_stl_file, World build),
// producing the flattened rt_scene_desc the device path consumes.
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/rtrace_gpu.h"

namespace rtb {

struct HostMesh {
  std::vector<double> vertices;  // 9 per triangle
  std::vector<rt_kd_node_desc> nodes;
  std::vector<int32_t> tri_index;
  double bmin[3], bmax[3];
};

// Owns every array an rt_scene_desc points to.
struct HostScene {
  rt_scene_desc desc{};
  std::vector<rt_object_desc> objects;
  std::vector<rt_material_desc> materials;
  std::vector<rt_light_desc> lights;
  std::vector<std::unique_ptr<HostMesh>> meshes;
  std::vector<rt_mesh_desc> mesh_descs;
  std::string render_error;
  void finalize();  // point desc at the owned arrays
};

// A k-d builder that runs elsewhere (on a device): KdTree::new(tris, 16, 10)
// over n triangles of 9 doubles each, with the host builder's preorder
// layout.  build returns "" on success, else the error that fails the load.
struct KdBuildHook {
  size_t min_triangles = 0;  // smaller meshes build on the host
  std::function<std::string(const double* vertices, size_t n, std::vector<rt_kd_node_desc>* nodes,
                            std::vector<int32_t>* idx)>
      build;
};

// Scene::from_json_str semantics with meshes resolved against base_dir
// ("" = current directory).  Returns false with *err set on failure.
bool load_scene_json(const std::string& text, const std::string& base_dir, HostScene* out, std::string* err,
                     const KdBuildHook* kd = nullptr);

// The host k-d builder (KdTree::new(tris, 16, 10), src/mesh.rs:75-197) over
// n triangles of 9 doubles each.  Returns "" or the reference's panic
// message for a NaN centre in a node it sorts.
std::string kd_build_host(const double* vertices, size_t n, std::vector<rt_kd_node_desc>* nodes,
                          std::vector<int32_t>* idx);
bool read_text_file(const std::string& path, std::string* out, std::string* err);
std::string parent_dir(const std::string& path);

// hex_to_color (src/scene.rs:15-30)
bool hex_to_color(const std::string& in, double out[3], std::string* err);

// Camera::from_config (src/camera.rs:23-153) output.
struct CameraBasis {
  double origin[3], horizontal[3], vertical[3], llc[3], view_dir[3];
  int persp;
  int grid_enabled;
  double grid_pitch, grid_half_thickness, grid_color[3];
};
bool make_camera(const rt_camera_config& cfg, double aspect, CameraBasis* out, std::string* err);

// AutoCamera::generate_cameras (src/auto_camera.rs:9-130): left, front, top
// and perspective views framing the scene's finite objects.
bool auto_cameras(const std::string& text, const std::string& base_dir, rt_camera_config out[4], std::string* err);

}  // namespace rtb
