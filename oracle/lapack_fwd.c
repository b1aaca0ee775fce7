/*
 * Test infrastructure only.  The reference's Ritz step calls LAPACK dsyev_
 * (include/sbd/framework/hp_numeric.h:497-517).  The only LAPACK in this image
 * is SciPy's bundled OpenBLAS, which exports the routine as scipy_dsyev_; this
 * forwarder gives the reference the symbol name it links against.
 */
extern void scipy_dsyev_(char*, char*, int*, double*, int*, double*, double*, int*, int*);

void dsyev_(char* jobz, char* uplo, int* n, double* a, int* lda, double* w, double* work,
            int* lwork, int* info) {
  scipy_dsyev_(jobz, uplo, n, a, lda, w, work, lwork, info);
}
