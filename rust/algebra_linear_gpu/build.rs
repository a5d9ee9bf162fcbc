//! Links libalgebra_linear_gpu.so. The library is built by the Python package
//! (`python -m algebra_linear_b200.build`), which writes it next to its
//! sources; ALGEBRA_LINEAR_GPU_LIB_DIR overrides the directory searched.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("ALGEBRA_LINEAR_GPU_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../../algebra_linear_b200"),
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=algebra_linear_gpu");
    println!("cargo:rerun-if-env-changed=ALGEBRA_LINEAR_GPU_LIB_DIR");
    println!("cargo:rerun-if-changed=../../include/algebra_linear_gpu.h");
}
