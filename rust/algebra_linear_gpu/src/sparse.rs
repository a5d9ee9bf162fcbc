//! The sparse LU handle with the reference's API
//! (`algebra_linear::sparse::faer::SparseLu<T>`, src/sparse/faer/sparse_lu.rs:45-156,
//! for `T` = `f64` or `Complex64`, lu.rs:20-82).
//! The symbolic analysis (COLAMD, elimination tree, column counts,
//! supernodes) runs on the host as the reference's does; every numeric
//! factorization and solve runs on the GPU. The caller owns the CSC arrays;
//! they are borrowed per call and never retained.

use core::ffi::c_int;
use core::marker::PhantomData;
use core::time::Duration;

use num_complex::Complex64;

use crate::ffi;

mod sealed {
    pub trait Sealed {}
    impl Sealed for f64 {}
    impl Sealed for num_complex::Complex64 {}
}

/// The scalars the sparse LU supports (the reference's `SparseScalar`,
/// lu.rs:20-82): `f64` and `Complex64` (`#[repr(C)]` (re, im), passed to the
/// library as interleaved doubles). Complex factors pivot by the modulus and
/// take their multipliers by `Complex::inv`, in FP64.
pub trait SparseScalar: Copy + sealed::Sealed {
    #[doc(hidden)]
    /// # Safety
    /// `h` is a live handle; the slices are valid for their lengths.
    unsafe fn factorize_raw(h: *mut ffi::alg_splu, col_ptr: &[usize], row_idx: &[usize], values: &[Self]) -> c_int;
    #[doc(hidden)]
    /// # Safety
    /// `h` is a live handle; `b` is valid for its length.
    unsafe fn solve_raw(h: *const ffi::alg_splu, b: &mut [Self]) -> c_int;
}

impl SparseScalar for f64 {
    unsafe fn factorize_raw(h: *mut ffi::alg_splu, col_ptr: &[usize], row_idx: &[usize], values: &[Self]) -> c_int {
        ffi::alg_splu_factorize(
            h,
            col_ptr.as_ptr(),
            col_ptr.len(),
            row_idx.as_ptr(),
            row_idx.len(),
            values.as_ptr(),
            values.len(),
        )
    }
    unsafe fn solve_raw(h: *const ffi::alg_splu, b: &mut [Self]) -> c_int {
        ffi::alg_splu_solve(h, b.as_mut_ptr(), b.len())
    }
}

impl SparseScalar for Complex64 {
    unsafe fn factorize_raw(h: *mut ffi::alg_splu, col_ptr: &[usize], row_idx: &[usize], values: &[Self]) -> c_int {
        ffi::alg_zsplu_factorize(
            h,
            col_ptr.as_ptr(),
            col_ptr.len(),
            row_idx.as_ptr(),
            row_idx.len(),
            values.as_ptr().cast::<f64>(),
            values.len(),
        )
    }
    unsafe fn solve_raw(h: *const ffi::alg_splu, b: &mut [Self]) -> c_int {
        ffi::alg_zsplu_solve(h, b.as_mut_ptr().cast::<f64>(), b.len())
    }
}

/// Errors reported by the sparse routines: the reference's `Error`
/// (src/sparse/faer/error.rs:5-24) in declaration order, plus [`Error::Device`]
/// for the conditions only a GPU has.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Error {
    BadShape,
    InvalidStructure,
    UnsortedRows,
    DuplicateEntry,
    Singular,
    IndexOverflow,
    StructureMismatch,
    NotFinite,
    NotFactorized,
    /// No counterpart in the reference: no usable device, a CUDA error, out
    /// of device memory or a timed-out device wait (the C ABI's status code).
    Device(i32),
}

impl core::fmt::Display for Error {
    fn fmt(&self, f: &mut core::fmt::Formatter<'_>) -> core::fmt::Result {
        // the reference's Display strings (error.rs:27-41)
        let msg = match self {
            Self::BadShape => "inconsistent shape or length",
            Self::InvalidStructure => "invalid CSC structure",
            Self::UnsortedRows => "row indices must be strictly increasing within a column",
            Self::DuplicateEntry => "duplicate entry in a column",
            Self::Singular => "the matrix is singular",
            Self::IndexOverflow => "index or workspace size overflow",
            Self::StructureMismatch => "the matrix pattern differs from the symbolic analysis",
            Self::NotFinite => "the matrix has a NaN or infinite entry",
            Self::NotFactorized => "the matrix has not been factorized",
            Self::Device(code) => crate::status_string(*code),
        };
        f.write_str(msg)
    }
}

impl std::error::Error for Error {}

fn map(rc: c_int) -> Result<(), Error> {
    Err(match rc {
        ffi::ALG_OK => return Ok(()),
        ffi::ALG_SP_BAD_SHAPE => Error::BadShape,
        ffi::ALG_SP_INVALID_STRUCTURE => Error::InvalidStructure,
        ffi::ALG_SP_UNSORTED_ROWS => Error::UnsortedRows,
        ffi::ALG_SP_DUPLICATE_ENTRY => Error::DuplicateEntry,
        ffi::ALG_SP_SINGULAR => Error::Singular,
        ffi::ALG_SP_INDEX_OVERFLOW => Error::IndexOverflow,
        ffi::ALG_SP_STRUCTURE_MISMATCH => Error::StructureMismatch,
        ffi::ALG_SP_NOT_FINITE => Error::NotFinite,
        ffi::ALG_SP_NOT_FACTORIZED => Error::NotFactorized,
        other => Error::Device(other),
    })
}

/// Which factorization the solver should use (solver.rs:71-96).
#[derive(Clone, Copy, Debug, PartialEq)]
pub enum LuMethod {
    Simplicial,
    Supernodal,
    /// Supernodal when `Σ col_counts² / nnz(A)` exceeds the threshold.
    Auto { flop_ratio_threshold: f64 },
}

impl LuMethod {
    /// The automatic method with the default threshold (`40.0`).
    pub fn auto() -> Self {
        Self::Auto { flop_ratio_threshold: 40.0 }
    }
}

impl Default for LuMethod {
    fn default() -> Self {
        Self::Simplicial
    }
}

/// The method selected by symbolic analysis (solver.rs:45-50).
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum EffectiveLuMethod {
    Simplicial,
    Supernodal,
}

/// Structure, cost and timing of a factorization (stats.rs:13-35).
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct SparseLuStats {
    pub n: usize,
    pub nnz_a: usize,
    /// Stored entries of `L`, including its unit diagonal.
    pub nnz_l: usize,
    pub nnz_u: usize,
    pub fill_ratio: f64,
    /// One multiply-add per `(L, U)` entry pair, summed over the columns.
    pub flops_estimate: usize,
    pub method: EffectiveLuMethod,
    pub flop_ratio: Option<f64>,
    pub ordering_time: Duration,
    pub factorization_time: Duration,
}

impl SparseLuStats {
    /// The stored entries of both factors.
    pub fn nnz_factors(&self) -> usize {
        self.nnz_l + self.nnz_u
    }
}

/// An opaque sparse LU factorization whose factors live on the GPU.
#[derive(Debug)]
pub struct SparseLu<T: SparseScalar = f64> {
    h: *mut ffi::alg_splu,
    n: usize,
    stats: Option<SparseLuStats>,
    _scalar: PhantomData<T>,
}

// The handle is used by one thread at a time (`&mut` for factorize), as the
// reference's is; moving it to another thread is fine.
unsafe impl<T: SparseScalar> Send for SparseLu<T> {}

impl<T: SparseScalar> SparseLu<T> {
    /// Analyzes the CSC pattern of a square matrix (sparse_lu.rs:64-78):
    /// `n = col_ptr.len() - 1`.
    ///
    /// # Errors
    ///
    /// [`Error::BadShape`] if `col_ptr` is empty or a row index is `>= n`,
    /// then the structural errors of the CSC validation.
    pub fn analyze(col_ptr: &[usize], row_idx: &[usize], method: LuMethod) -> Result<Self, Error> {
        let n = col_ptr.len().checked_sub(1).ok_or(Error::BadShape)?;
        let (m, thr) = match method {
            LuMethod::Simplicial => (ffi::ALG_SPLU_SIMPLICIAL, 40.0),
            LuMethod::Supernodal => (ffi::ALG_SPLU_SUPERNODAL, 40.0),
            LuMethod::Auto { flop_ratio_threshold } => (ffi::ALG_SPLU_AUTO, flop_ratio_threshold),
        };
        let mut h = core::ptr::null_mut();
        // SAFETY: the slices are valid for their lengths for the call.
        map(unsafe {
            ffi::alg_splu_analyze(col_ptr.as_ptr(), col_ptr.len(), row_idx.as_ptr(), row_idx.len(), m, thr, &mut h)
        })?;
        Ok(Self { h, n, stats: None, _scalar: PhantomData })
    }

    /// Factorizes new values on the analyzed pattern (sparse_lu.rs:91-121).
    /// A failed factorization leaves the previous factors and statistics in
    /// place.
    ///
    /// # Errors
    ///
    /// The CSC view errors, then [`Error::StructureMismatch`],
    /// [`Error::NotFinite`] (either part, for complex values), [`Error::Singular`].
    pub fn factorize(&mut self, col_ptr: &[usize], row_idx: &[usize], values: &[T]) -> Result<(), Error> {
        // SAFETY: the handle is live and the slices are valid for their lengths for the call.
        map(unsafe { T::factorize_raw(self.h, col_ptr, row_idx, values) })?;
        // SAFETY: a plain C struct, filled by the library.
        let mut s: ffi::alg_splu_stats = unsafe { core::mem::zeroed() };
        map(unsafe { ffi::alg_splu_get_stats(self.h, &mut s) })?;
        self.stats = Some(SparseLuStats {
            n: s.n,
            nnz_a: s.nnz_a,
            nnz_l: s.nnz_l,
            nnz_u: s.nnz_u,
            fill_ratio: s.fill_ratio,
            flops_estimate: s.flops_estimate,
            method: if s.method == ffi::ALG_SPLU_SUPERNODAL {
                EffectiveLuMethod::Supernodal
            } else {
                EffectiveLuMethod::Simplicial
            },
            flop_ratio: if s.has_flop_ratio != 0 { Some(s.flop_ratio) } else { None },
            ordering_time: Duration::from_secs_f64(s.ordering_time.max(0.0)),
            factorization_time: Duration::from_secs_f64(s.factorization_time.max(0.0)),
        });
        Ok(())
    }

    /// Solves `A x = b` in place (sparse_lu.rs:125-130).
    ///
    /// # Errors
    ///
    /// [`Error::NotFactorized`] before a successful factorization,
    /// [`Error::BadShape`] if `b.len() != n`.
    pub fn solve(&self, b: &mut [T]) -> Result<(), Error> {
        // SAFETY: the handle is live and b is valid for its length for the call.
        map(unsafe { T::solve_raw(self.h, b) })
    }

    /// The method selected during analysis (sparse_lu.rs:137-140).
    pub fn effective_method(&self) -> EffectiveLuMethod {
        // SAFETY: the handle is valid until drop.
        if unsafe { ffi::alg_splu_effective_method(self.h) } == ffi::ALG_SPLU_SUPERNODAL {
            EffectiveLuMethod::Supernodal
        } else {
            EffectiveLuMethod::Simplicial
        }
    }

    /// The flop-ratio proxy, when the supernodal analysis ran (sparse_lu.rs:146-149).
    pub fn flop_ratio(&self) -> Option<f64> {
        let mut r = 0.0;
        // SAFETY: the handle is valid until drop.
        if unsafe { ffi::alg_splu_flop_ratio(self.h, &mut r) } != 0 {
            Some(r)
        } else {
            None
        }
    }

    /// Statistics of the last successful factorization (sparse_lu.rs:152-155).
    pub fn stats(&self) -> Option<&SparseLuStats> {
        self.stats.as_ref()
    }

    /// The order of the matrix.
    pub fn n(&self) -> usize {
        self.n
    }
}

impl<T: SparseScalar> Drop for SparseLu<T> {
    fn drop(&mut self) {
        // SAFETY: the handle came from alg_splu_analyze and is freed once.
        unsafe { ffi::alg_splu_free(self.h) };
    }
}
