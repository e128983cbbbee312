/*
 * Build helper for oracle/_ref (test infrastructure only).
 *
 * The reference's C library (src/bdsim/clib/diff_tensor.c:22-25) calls the
 * Fortran LAPACK symbols dgetrf_/dgetri_.  No system LAPACK exists in this
 * image, so these two forwarders route the calls to the LP64 LAPACK that
 * SciPy ships (its exported names carry a "scipy_" prefix).
 */
void scipy_dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info);
void scipy_dgetri_(int *n, double *a, int *lda, int *ipiv, double *work, int *lwork, int *info);

void dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info)
{
	scipy_dgetrf_(m, n, a, lda, ipiv, info);
}

void dgetri_(int *n, double *a, int *lda, int *ipiv, double *work, int *lwork, int *info)
{
	scipy_dgetri_(n, a, lda, ipiv, work, lwork, info);
}
