//! Links the static CUDA library of this repository (`toaster_b200/lib/libtoaster_cuda.a`, built by
//! `python -m toaster_b200.build`) and the CUDA runtime it needs.
//!
//! `TOASTER_CUDA_LIB_DIR` names the directory holding `libtoaster_cuda.a`; `CUDA_PATH` the CUDA
//! installation (default `/usr/local/cuda`).

fn main() {
    let lib = std::env::var("TOASTER_CUDA_LIB_DIR")
        .expect("TOASTER_CUDA_LIB_DIR must name the directory of libtoaster_cuda.a");
    let cuda = std::env::var("CUDA_PATH").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rerun-if-env-changed=TOASTER_CUDA_LIB_DIR");
    println!("cargo:rerun-if-env-changed=CUDA_PATH");
    println!("cargo:rerun-if-changed={lib}/libtoaster_cuda.a");
    println!("cargo:rustc-link-search=native={lib}");
    println!("cargo:rustc-link-lib=static=toaster_cuda");
    println!("cargo:rustc-link-search=native={cuda}/lib64");
    println!("cargo:rustc-link-lib=static=cudart_static");
    println!("cargo:rustc-link-lib=dylib=nvjpeg"); // tc_encode_jpeg
    println!("cargo:rustc-link-lib=dylib=z"); // PNG textures in tc_scene_load
    println!("cargo:rustc-link-lib=dylib=stdc++");
    println!("cargo:rustc-link-lib=dylib=rt");
    println!("cargo:rustc-link-lib=dylib=dl");
    println!("cargo:rustc-link-lib=dylib=pthread");
}
