//! Safe Rust bindings of `libalgebra_linear_gpu`, the B200 (sm_100a) LU
//! solver, with the signatures of the dense and sparse LU path of the
//! `algebra_linear` 4.0.0 crate, so a caller switches by changing the path
//! it imports:
//!
//! | `algebra_linear` | here |
//! |---|---|
//! | `lapack::dgetrf` (src/lapack/mod.rs:181) | [`lapack::dgetrf`] |
//! | `lapack::dgetrf_rect` (mod.rs:202) | [`lapack::dgetrf_rect`] |
//! | `lapack::dgesv` (mod.rs:309) | [`lapack::dgesv`] |
//! | `lapack::dgetri` (mod.rs:249) | [`lapack::dgetri`] |
//! | `lapack::zgetrf` / `zgetrf_rect` / `zgesv` / `zgetri` (complex.rs:67, 169, 279, 217) | [`complex`] |
//! | `sparse::faer::SparseLu<f64>`, `SparseLu<Complex64>` (sparse_lu.rs:45-156, lu.rs:20-82) | [`sparse::SparseLu`] |
//!
//! Errors are the reference's enums ([`LapackError`], [`sparse::Error`]); a
//! condition only a GPU has (no device, a CUDA error, out of device memory, a
//! timed-out device wait) is reported as [`LapackError::NotImplemented`] with
//! the library's message by the dense routines and as [`sparse::Error::Device`]
//! (the one variant the reference's sparse `Error` lacks) by the sparse handle.
//!
//! The raw declarations are in [`ffi`], written from the C header by
//! `gen_ffi.py`. Beyond the reference's API, [`lapack::dgesv_mixed`] exposes
//! the mixed-precision solve (FP32 LU on the tensor cores + FP64 refinement
//! to the FP64 backward error).

pub mod complex;
pub mod ffi;
pub mod lapack;
pub mod sparse;

pub use lapack::LapackError;

/// The library's message for a status code.
pub fn status_string(status: core::ffi::c_int) -> &'static str {
    // SAFETY: the library returns a pointer to static storage for every code.
    unsafe {
        let p = ffi::alg_status_string(status);
        if p.is_null() {
            return "unknown status";
        }
        core::ffi::CStr::from_ptr(p).to_str().unwrap_or("unknown status")
    }
}
