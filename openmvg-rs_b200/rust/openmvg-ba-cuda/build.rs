// Links libomvgba_cuda.so, built by openmvg-rs_b200/build.py (nvcc, sm_100a). The directory comes
// from OMVGBA_CUDA_LIB_DIR; the library needs the CUDA runtime at run time.
fn main() {
    let dir = std::env::var("OMVGBA_CUDA_LIB_DIR")
        .expect("set OMVGBA_CUDA_LIB_DIR to the directory holding libomvgba_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=omvgba_cuda");
    println!("cargo:rerun-if-env-changed=OMVGBA_CUDA_LIB_DIR");
}
