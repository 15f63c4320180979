//! Rust binding of the B200 render path's C ABI (include/rtrace_gpu.h).
//!
//! Not compiled in this repository: its image has no Rust toolchain.  The
//! `ffi` module mirrors the header's structs and the entry points the
//! reference's front ends need; `GpuRenderer` is the safe layer they call.
//!
//! Where it plugs in (the reference's own files):
//! - cli/src/main.rs:358-402 calls `Renderer::render_to_file(&scene, output)`
//!   after `Scene::from_json_file(input)`; with this crate it calls
//!   `GpuRenderer::render_file_to_png(&renderer_fields, input, output)`.
//! - bindings/node/src/lib.rs:17-318: `render_scene*` take a JSON string and
//!   call `Scene::from_json_str` (meshes relative to "."), the
//!   `render_scene_from_file*` variants a path; they call `render_json_str`
//!   and `render_json_file` instead, with the same `Status::InvalidArg` for
//!   parse errors (`RtError::Scene`) and `Status::GenericFailure` for render
//!   errors.
//! - src/renderer.rs:120 `Renderer::render(&self, &Scene)`: a scene already
//!   parsed in Rust is serialised back (`Scene` derives `Serialize`) and
//!   loaded by the C++ loader; its meshes resolve relative to the current
//!   directory, as `Scene::from_json_str` resolves them.
//!
//! Errors carry the reference's own messages ("Samples must be greater than
//! 0", "Field of view must be between 0 and 180 degrees", "Unsupported
//! camera type: ...", "Invalid hex color ...").

use std::ffi::{CStr, CString};
use std::os::raw::c_int;

pub mod ffi {
    use std::os::raw::{c_char, c_int};

    #[repr(C)]
    pub struct RtCtx {
        _p: [u8; 0],
    }
    #[repr(C)]
    pub struct RtScene {
        _p: [u8; 0],
    }
    #[repr(C)]
    pub struct RtHostScene {
        _p: [u8; 0],
    }

    pub const RT_OK: c_int = 0;
    pub const RT_ERR_INVALID_ARGUMENT: c_int = 1;
    pub const RT_ERR_SCENE: c_int = 2;
    pub const RT_ERR_RENDER: c_int = 3;
    pub const RT_ERR_IO: c_int = 7;

    pub const RT_AA_NO_JITTER: i32 = 0;
    pub const RT_AA_QUINCUNX: i32 = 1;
    pub const RT_AA_STOCHASTIC: i32 = 2;
    pub const RT_STAGE_COUNT: usize = 8;

    /// rt_outline_config: OutlineConfig (src/outline.rs:5-31).
    #[repr(C)]
    #[derive(Default, Clone, Copy, Debug)]
    pub struct RtOutlineConfig {
        pub enabled: i32,
        pub use_8_neighbors: i32,
        pub depth_weight: f64,
        pub normal_weight: f64,
        pub threshold: f64,
        pub edge_color: [f64; 3],
        pub line_thickness: f64,
        /// extension: edges between different objects (0: the reference's outline)
        pub object_id_weight: f64,
    }

    /// rt_render_params: the Renderer fields (src/renderer.rs:37-47) and the
    /// extensions, whose zero values keep the reference's behaviour.
    #[repr(C)]
    #[derive(Default, Clone, Copy, Debug)]
    pub struct RtRenderParams {
        pub width: u32,
        pub height: u32,
        pub max_depth: i32,
        pub use_kdtree: i32,
        pub samples: u32,
        pub anti_aliasing_mode: i32,
        pub seed: u64,
        pub outline: RtOutlineConfig,
        pub flags: u32,
        pub reserved: u32,
        pub disk_samples: u32,
        pub learned_shadows: i32,
        pub learned_rays: u32,
        pub fallback_samples: u32,
        pub confidence_threshold: f32,
        pub reserved3: u32,
    }

    /// rt_stats
    #[repr(C)]
    #[derive(Default, Clone, Copy, Debug)]
    pub struct RtStats {
        pub primary_rays: u64,
        pub reflection_rays: u64,
        pub shadow_rays: u64,
        pub hits: u64,
        pub trace_nodes: u64,
        pub trace_triangles: u64,
        pub trace_spheres: u64,
        pub trace_verifications: u64,
        pub shadow_nodes: u64,
        pub shadow_triangles: u64,
        pub shadow_spheres: u64,
        pub shadow_verifications: u64,
        pub kernel_launches: u32,
        pub graph: u32,
        pub device_ms: f64,
        pub total_ms: f64,
        pub stage_ms: [f64; RT_STAGE_COUNT],
        pub fallback_hits: u64,
        pub fallback_lights: u64,
        pub shadow_rays_untraced: u64,
    }

    extern "C" {
        pub fn rt_ctx_create(device: c_int, out: *mut *mut RtCtx) -> c_int;
        pub fn rt_ctx_destroy(ctx: *mut RtCtx);
        pub fn rt_last_error(ctx: *const RtCtx) -> *const c_char;
        pub fn rt_host_scene_load_json_file_on(ctx: *mut RtCtx, path: *const c_char, out: *mut *mut RtHostScene)
            -> c_int;
        pub fn rt_host_scene_load_json_str_on(ctx: *mut RtCtx, json: *const c_char, out: *mut *mut RtHostScene)
            -> c_int;
        pub fn rt_host_scene_upload(ctx: *mut RtCtx, hs: *mut RtHostScene, out: *mut *mut RtScene) -> c_int;
        pub fn rt_host_scene_free(hs: *mut RtHostScene);
        pub fn rt_scene_free(scene: *mut RtScene);
        pub fn rt_scene_outline_config(ctx: *mut RtCtx, scene: *const RtScene, out: *mut RtOutlineConfig) -> c_int;
        pub fn rt_scene_camera_aspect(ctx: *mut RtCtx, scene: *const RtScene, out: *mut f64) -> c_int;
        pub fn rt_render(ctx: *mut RtCtx, scene: *const RtScene, params: *const RtRenderParams, rgb_out: *mut u8,
                         out_on_device: c_int, stats: *mut RtStats) -> c_int;
        pub fn rt_png_write(path: *const c_char, rgb: *const u8, width: u32, height: u32) -> c_int;
        pub fn rt_denoiser_load(ctx: *mut RtCtx, blob: *const u8, bytes: usize) -> c_int;
    }
}

/// Errors of the GPU path, with the reference's messages.
#[derive(Debug)]
pub enum RtError {
    /// Scene::from_json_* failed (the napi bindings map it to InvalidArg).
    Scene(String),
    /// Renderer::render failed (GenericFailure in the napi bindings).
    Render(String),
    /// Bad arguments, CUDA, memory or I/O failures the reference cannot have.
    Device(String),
}

impl std::fmt::Display for RtError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        match self {
            RtError::Scene(m) | RtError::Render(m) | RtError::Device(m) => f.write_str(m),
        }
    }
}
impl std::error::Error for RtError {}

/// The Renderer fields the GPU path needs (src/renderer.rs:37-47).
#[derive(Clone, Debug)]
pub struct RenderSettings {
    pub width: u32,
    pub height: u32,
    pub max_depth: i32,
    pub use_kdtree: bool,
    pub samples: u32,
    /// 0 no-jitter, 1 quincunx (the reference's default), 2 stochastic
    pub anti_aliasing_mode: i32,
    pub seed: Option<u64>,
    /// Some(..) enables the outline (ignored in quincunx, as the reference does)
    pub outline: Option<ffi::RtOutlineConfig>,
}

/// One CUDA device's context.  The reference's `Renderer::render` takes
/// `&self` and is re-entrant; a context is not: keep one per thread.
pub struct GpuRenderer {
    ctx: *mut ffi::RtCtx,
}

unsafe impl Send for GpuRenderer {}

fn last_error(ctx: *const ffi::RtCtx) -> String {
    unsafe {
        let p = ffi::rt_last_error(ctx);
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

fn check(ctx: *const ffi::RtCtx, st: c_int) -> Result<(), RtError> {
    match st {
        ffi::RT_OK => Ok(()),
        ffi::RT_ERR_SCENE => Err(RtError::Scene(last_error(ctx))),
        ffi::RT_ERR_RENDER => Err(RtError::Render(last_error(ctx))),
        _ => Err(RtError::Device(last_error(ctx))),
    }
}

impl GpuRenderer {
    pub fn new(device: i32) -> Result<Self, RtError> {
        let mut ctx = std::ptr::null_mut();
        check(std::ptr::null(), unsafe { ffi::rt_ctx_create(device as c_int, &mut ctx) })?;
        Ok(GpuRenderer { ctx })
    }

    fn params(&self, s: &RenderSettings) -> ffi::RtRenderParams {
        ffi::RtRenderParams {
            width: s.width,
            height: s.height,
            max_depth: s.max_depth,
            use_kdtree: s.use_kdtree as i32,
            samples: s.samples,
            anti_aliasing_mode: s.anti_aliasing_mode,
            seed: s.seed.unwrap_or(0),
            outline: s.outline.unwrap_or_default(),
            ..Default::default()
        }
    }

    fn render_host_scene(&self, hs: *mut ffi::RtHostScene, s: &RenderSettings) -> Result<Vec<u8>, RtError> {
        let mut scene = std::ptr::null_mut();
        let st = unsafe { ffi::rt_host_scene_upload(self.ctx, hs, &mut scene) };
        unsafe { ffi::rt_host_scene_free(hs) };
        check(self.ctx, st)?;
        let params = self.params(s);
        let mut rgb = vec![0u8; s.width as usize * s.height as usize * 3];
        let st = unsafe {
            ffi::rt_render(self.ctx, scene, &params, rgb.as_mut_ptr(), 0, std::ptr::null_mut())
        };
        unsafe { ffi::rt_scene_free(scene) };
        check(self.ctx, st)?;
        Ok(rgb)
    }

    /// Scene::from_json_file + Renderer::render: RGB8, width*height*3 bytes.
    pub fn render_json_file(&self, path: &str, s: &RenderSettings) -> Result<Vec<u8>, RtError> {
        let c = CString::new(path).map_err(|e| RtError::Scene(e.to_string()))?;
        let mut hs = std::ptr::null_mut();
        check(self.ctx, unsafe { ffi::rt_host_scene_load_json_file_on(self.ctx, c.as_ptr(), &mut hs) })?;
        self.render_host_scene(hs, s)
    }

    /// Scene::from_json_str (meshes relative to ".") + Renderer::render.
    pub fn render_json_str(&self, json: &str, s: &RenderSettings) -> Result<Vec<u8>, RtError> {
        let c = CString::new(json).map_err(|e| RtError::Scene(e.to_string()))?;
        let mut hs = std::ptr::null_mut();
        check(self.ctx, unsafe { ffi::rt_host_scene_load_json_str_on(self.ctx, c.as_ptr(), &mut hs) })?;
        self.render_host_scene(hs, s)
    }

    /// The same, wrapped in the `RgbImage` Renderer::render returns.
    pub fn render_json_file_image(&self, path: &str, s: &RenderSettings) -> Result<image::RgbImage, RtError> {
        let rgb = self.render_json_file(path, s)?;
        image::RgbImage::from_raw(s.width, s.height, rgb).ok_or_else(|| RtError::Device("image size".into()))
    }

    /// Renderer::render_to_file (src/renderer.rs:914-920) for the CLI: the
    /// PNG is encoded on the host's threads (rt_png_write).
    pub fn render_file_to_png(&self, s: &RenderSettings, input: &str, output: &str) -> Result<(), RtError> {
        let rgb = self.render_json_file(input, s)?;
        let c = CString::new(output).map_err(|e| RtError::Device(e.to_string()))?;
        check(self.ctx, unsafe { ffi::rt_png_write(c.as_ptr(), rgb.as_ptr(), s.width, s.height) })
    }

    /// Loads the learned soft-shadow denoiser (extension): the bytes of
    /// rtrace_b200/denoiser_weights.bin.
    pub fn load_denoiser(&self, blob: &[u8]) -> Result<(), RtError> {
        check(self.ctx, unsafe { ffi::rt_denoiser_load(self.ctx, blob.as_ptr(), blob.len()) })
    }
}

impl Drop for GpuRenderer {
    fn drop(&mut self) {
        unsafe { ffi::rt_ctx_destroy(self.ctx) };
    }
}

/// The body a maintainer gives `Renderer::render` (src/renderer.rs:120):
/// the parsed scene goes back to JSON (it derives Serialize) and through
/// the C++ loader; meshes resolve relative to the current directory.
pub fn render_scene_json(gpu: &GpuRenderer, scene_json: &str, s: &RenderSettings) -> Result<Vec<u8>, RtError> {
    gpu.render_json_str(scene_json, s)
}
