// Links librtrace_b200.so (sm_100a), built by `python -m rtrace_b200.build`
// into rtrace_b200/_lib.  Not built in this repository (no Rust toolchain).
fn main() {
    let dir = std::env::var("RTRACE_GPU_LIB_DIR").unwrap_or_else(|_| "../../rtrace_b200/_lib".to_string());
    println!("cargo:rustc-link-search=native={}", dir);
    println!("cargo:rustc-link-lib=dylib=rtrace_b200");
    println!("cargo:rerun-if-env-changed=RTRACE_GPU_LIB_DIR");
}
