//! The dense LU routines with the reference's signatures
//! (`algebra_linear::lapack`, src/lapack/mod.rs). Each call copies the
//! caller's slices to the GPU, computes there and copies the results back
//! into the same slices, as the reference computes in place.

use core::ffi::c_int;

use crate::ffi;

/// Error kinds these routines can report (the reference's `LapackError`,
/// src/lapack/mod.rs:76-96, variant for variant).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum LapackError {
    /// The matrix is singular to working precision (a zero pivot).
    Singular,
    /// A shape or length was inconsistent with another.
    BadShape,
    /// An iterative routine exhausted its iteration limit before converging.
    Convergence,
    /// Carries a name or message; here, a condition only the GPU has (no
    /// device, a CUDA error, out of device memory, a timed-out device wait).
    NotImplemented(&'static str),
}

impl core::fmt::Display for LapackError {
    fn fmt(&self, f: &mut core::fmt::Formatter<'_>) -> core::fmt::Result {
        match self {
            Self::Singular => f.write_str("the matrix is singular"),
            Self::BadShape => f.write_str("inconsistent shape or length"),
            Self::Convergence => f.write_str("the iteration did not converge"),
            Self::NotImplemented(what) => write!(f, "{what}"),
        }
    }
}

impl std::error::Error for LapackError {}

pub(crate) fn map(rc: c_int) -> Result<(), LapackError> {
    match rc {
        ffi::ALG_OK => Ok(()),
        ffi::ALG_SINGULAR => Err(LapackError::Singular),
        ffi::ALG_BAD_SHAPE => Err(LapackError::BadShape),
        ffi::ALG_CONVERGENCE => Err(LapackError::Convergence),
        other => Err(LapackError::NotImplemented(crate::status_string(other))),
    }
}

/// `dgetrf`: LU factorization with partial pivoting, in place
/// (src/lapack/mod.rs:181-185). Returns the 0-based sequential interchanges
/// and the determinant. The factors, pivots and determinant are
/// bit-identical to the reference's.
///
/// # Errors
///
/// [`LapackError::BadShape`] if `a.len() != n * n`; [`LapackError::Singular`]
/// on a zero pivot (then `a` is unspecified, as the reference leaves it
/// partly factored).
pub fn dgetrf(a: &mut [f64], n: usize) -> Result<(Vec<usize>, f64), LapackError> {
    if n.checked_mul(n) != Some(a.len()) {
        return Err(LapackError::BadShape);
    }
    let mut ipiv = vec![0usize; n];
    let mut det = 1.0;
    if n == 0 {
        return Ok((ipiv, det));
    }
    // SAFETY: a holds n * n values and ipiv n entries, as the C ABI requires.
    map(unsafe { ffi::alg_dgetrf(a.as_mut_ptr(), n, ipiv.as_mut_ptr(), &mut det) })?;
    Ok((ipiv, det))
}

/// `dgetrf_rect`: LU with partial pivoting of an `nrows x ncols` panel
/// (`nrows >= ncols`), interchanges within its columns
/// (src/lapack/mod.rs:202-238).
///
/// # Errors
///
/// [`LapackError::BadShape`] if `nrows < ncols` or the lengths disagree;
/// [`LapackError::Singular`] on a zero pivot.
pub fn dgetrf_rect(a: &mut [f64], nrows: usize, ncols: usize, ipiv: &mut [usize]) -> Result<(), LapackError> {
    if nrows < ncols || nrows.checked_mul(ncols) != Some(a.len()) || ipiv.len() != ncols {
        return Err(LapackError::BadShape);
    }
    if ncols == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_dgetrf_rect(a.as_mut_ptr(), nrows, ncols, ipiv.as_mut_ptr()) })
}

/// `dgesv`: solves `A x = b` with `n = b.len()` (src/lapack/mod.rs:309-323).
/// `a` is left holding its LU factors and `b` holds `x`.
///
/// # Errors
///
/// [`LapackError::BadShape`] if `a.len() != n * n`; [`LapackError::Singular`]
/// on a zero pivot.
pub fn dgesv(a: &mut [f64], b: &mut [f64]) -> Result<(), LapackError> {
    let n = b.len();
    if n.checked_mul(n) != Some(a.len()) {
        return Err(LapackError::BadShape);
    }
    if n == 0 {
        return Ok(());
    }
    // SAFETY: a holds n * n values and b n values.
    map(unsafe { ffi::alg_dgesv(a.as_mut_ptr(), b.as_mut_ptr(), n) })
}

/// `dgesv` with several right-hand sides: `b` is `n x nrhs` column-major;
/// each column is solved as the reference's `dgetrs`.
///
/// # Errors
///
/// [`LapackError::BadShape`] if `a.len() != n * n` or `b.len() != n * nrhs`.
pub fn dgesv_nrhs(a: &mut [f64], b: &mut [f64], n: usize, nrhs: usize) -> Result<(), LapackError> {
    if n.checked_mul(n) != Some(a.len()) || n.checked_mul(nrhs) != Some(b.len()) {
        return Err(LapackError::BadShape);
    }
    if n == 0 || nrhs == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_dgesv_nrhs(a.as_mut_ptr(), b.as_mut_ptr(), n, nrhs) })
}

/// `dgetri`: the inverse from the factors and pivots of [`dgetrf`]
/// (src/lapack/mod.rs:249-298), bit-identical to the reference's.
///
/// # Errors
///
/// [`LapackError::BadShape`] on inconsistent lengths or a pivot out of
/// range; [`LapackError::Singular`] when some `u_ii` is zero (`lu` unchanged).
pub fn dgetri(lu: &mut [f64], n: usize, ipiv: &[usize]) -> Result<(), LapackError> {
    if n.checked_mul(n) != Some(lu.len()) || ipiv.len() != n {
        return Err(LapackError::BadShape);
    }
    if n == 0 {
        return Ok(());
    }
    // SAFETY: the lengths were checked above.
    map(unsafe { ffi::alg_dgetri(lu.as_mut_ptr(), n, ipiv.as_ptr()) })
}

/// Precision of the mixed solve's LU (trailing updates; FP32 accumulation).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum MixedPrecision {
    /// FP32 on the CUDA cores.
    Fp32,
    /// TF32 on the tensor cores.
    Tf32,
    /// BF16 on the tensor cores.
    Bf16,
    /// FP32 operands split into TF32 pairs, three tensor-core products.
    Tf32x3,
}

/// How the mixed solve ended.
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct MixedReport {
    /// 1: refinement, 2: GMRES-IR, 3: the FP64 fallback refactorization.
    pub path: i32,
    pub ir_iterations: i32,
    pub gmres_iterations: i32,
    /// Normwise backward error of x (worst over the right-hand sides; -1 on
    /// the FP64 fallback).
    pub backward_error: f64,
}

/// Mixed-precision `dgesv` (no counterpart in the reference): a
/// low-precision LU refined in FP64 until the normwise backward error is
/// within `10 n 2^-53`, the FP64 level. `a` is left unchanged unless the FP64
/// fallback ran (then it holds the FP64 LU, as after [`dgesv`]); `b`
/// (`n x nrhs`) becomes `x`.
///
/// # Errors
///
/// [`LapackError::BadShape`] on inconsistent lengths; [`LapackError::Singular`]
/// if the FP64 fallback meets a zero pivot.
pub fn dgesv_mixed(
    a: &mut [f64],
    b: &mut [f64],
    n: usize,
    nrhs: usize,
    precision: MixedPrecision,
) -> Result<MixedReport, LapackError> {
    if n.checked_mul(n) != Some(a.len()) || n.checked_mul(nrhs) != Some(b.len()) {
        return Err(LapackError::BadShape);
    }
    // SAFETY: plain C structs, filled by the library.
    let mut opts: ffi::alg_mixed_opts = unsafe { core::mem::zeroed() };
    let mut rep: ffi::alg_mixed_report = unsafe { core::mem::zeroed() };
    unsafe { ffi::alg_mixed_opts_default(&mut opts) };
    opts.precision = match precision {
        MixedPrecision::Fp32 => ffi::ALG_PREC_FP32,
        MixedPrecision::Tf32 => ffi::ALG_PREC_TF32,
        MixedPrecision::Bf16 => ffi::ALG_PREC_BF16,
        MixedPrecision::Tf32x3 => ffi::ALG_PREC_TF32X3,
    };
    if n > 0 && nrhs > 0 {
        // SAFETY: the lengths were checked above.
        map(unsafe { ffi::alg_dgesv_mixed(&opts, a.as_mut_ptr(), b.as_mut_ptr(), n, nrhs, &mut rep) })?;
    }
    Ok(MixedReport {
        path: rep.path,
        ir_iterations: rep.ir_iterations,
        gmres_iterations: rep.gmres_iterations,
        backward_error: rep.backward_error,
    })
}
