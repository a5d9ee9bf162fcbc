//! The complex dense LU twins with the reference's signatures
//! (`algebra_linear::lapack::{zgetrf, zgetrf_rect, zgesv, zgetri}`,
//! src/lapack/complex.rs). `Complex64` is `#[repr(C)]` (re, im), the
//! interleaved layout the C ABI takes, so slices are passed as they are.
//! Results are bit-identical to the reference's (|Re| + |Im| pivots,
//! num-complex 0.4 arithmetic with every operation rounded on its own).

use num_complex::Complex64;

use crate::ffi;
use crate::lapack::{map, LapackError};

fn as_f64(a: &mut [Complex64]) -> *mut f64 {
    a.as_mut_ptr().cast::<f64>()
}

/// `zgetrf` (complex.rs:67-124): in-place LU with partial pivoting;
/// returns the 0-based interchanges.
///
/// # Errors
///
/// [`LapackError::BadShape`] if `a.len() != n * n`; [`LapackError::Singular`]
/// on a zero pivot.
pub fn zgetrf(a: &mut [Complex64], n: usize) -> Result<Vec<usize>, LapackError> {
    if n.checked_mul(n) != Some(a.len()) {
        return Err(LapackError::BadShape);
    }
    let mut ipiv = vec![0usize; n];
    if n == 0 {
        return Ok(ipiv);
    }
    // SAFETY: a holds n * n complex values (2 n^2 doubles), ipiv n entries.
    map(unsafe { ffi::alg_zgetrf(as_f64(a), n, ipiv.as_mut_ptr()) })?;
    Ok(ipiv)
}

/// `zgetrf_rect` (complex.rs:169-208): LU of an `nrows x ncols` panel.
///
/// # Errors
///
/// [`LapackError::BadShape`] if the lengths disagree or `nrows < ncols`;
/// [`LapackError::Singular`] on a zero pivot.
pub fn zgetrf_rect(a: &mut [Complex64], nrows: usize, ncols: usize, ipiv: &mut [usize]) -> Result<(), LapackError> {
    if nrows < ncols || nrows.checked_mul(ncols) != Some(a.len()) || ipiv.len() != ncols {
        return Err(LapackError::BadShape);
    }
    if ncols == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_zgetrf_rect(as_f64(a), nrows, ncols, ipiv.as_mut_ptr()) })
}

/// `zgesv` (complex.rs:279-312): `n = b.len()`; `a` keeps its LU factors,
/// `b` becomes `x`.
///
/// # Errors
///
/// [`LapackError::BadShape`] if `a.len() != n * n`; [`LapackError::Singular`]
/// on a zero pivot.
pub fn zgesv(a: &mut [Complex64], b: &mut [Complex64]) -> Result<(), LapackError> {
    let n = b.len();
    if n.checked_mul(n) != Some(a.len()) {
        return Err(LapackError::BadShape);
    }
    if n == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_zgesv(as_f64(a), as_f64(b), n) })
}

/// `zgetri` (complex.rs:217-271): the inverse from the factors and pivots of
/// [`zgetrf`].
///
/// # Errors
///
/// [`LapackError::BadShape`] if the shapes disagree or a pivot is out of
/// range; [`LapackError::Singular`] on a zero `u_jj`.
pub fn zgetri(lu: &mut [Complex64], n: usize, ipiv: &[usize]) -> Result<(), LapackError> {
    if n.checked_mul(n) != Some(lu.len()) || ipiv.len() != n {
        return Err(LapackError::BadShape);
    }
    if n == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_zgetri(as_f64(lu), n, ipiv.as_ptr()) })
}
