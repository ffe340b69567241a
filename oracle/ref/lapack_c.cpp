// dgesv_ for the reference's bilinear interpolation (src/adjoint/bilinear_interp.C:350-392), which
// calls LAPACK to solve one 4 x 4 system per interpolated value.  LAPACK is a third-party library
// the harness does not link (not installed here); this is a restatement of its published
// algorithm (LAPACK 3.x dgesv = dgetrf + dgetrs): LU factorisation with partial pivoting in the
// unblocked right-looking order of dgetf2 (pivot = the first entry of largest magnitude in the
// column, row swap, the column below the pivot scaled by the pivot's reciprocal, rank-1 update of
// the trailing block), then the row interchanges on the right-hand sides and the unit-lower and
// upper triangular solves of dgetrs.  Column-major, 1-based pivot indices, info > 0 on a zero
// pivot.  Test infrastructure only; its results can differ from a tuned LAPACK in the last bits.
#include <cmath>

extern "C" void dgesv_(int *n_, int *nrhs_, double *a, int *lda_, int *ipiv, double *b, int *ldb_, int *info) {
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    *info = 0;
    auto A = [&](int i, int j) -> double & { return a[i + (long)j * lda]; };
    for (int j = 0; j < n; ++j) {
        int p = j;
        double best = std::fabs(A(j, j));
        for (int i = j + 1; i < n; ++i)
            if (std::fabs(A(i, j)) > best) {
                best = std::fabs(A(i, j));
                p = i;
            }
        ipiv[j] = p + 1;
        if (A(p, j) == 0.0) {
            if (*info == 0) *info = j + 1;
            continue;
        }
        if (p != j)
            for (int k = 0; k < n; ++k) {
                const double t = A(j, k);
                A(j, k) = A(p, k);
                A(p, k) = t;
            }
        const double r = 1.0 / A(j, j);
        for (int i = j + 1; i < n; ++i) A(i, j) *= r;
        for (int k = j + 1; k < n; ++k) {
            const double t = A(j, k);
            if (t != 0.0)
                for (int i = j + 1; i < n; ++i) A(i, k) -= A(i, j) * t;
        }
    }
    if (*info) return;
    for (int c = 0; c < nrhs; ++c) {
        double *x = b + (long)c * ldb;
        for (int j = 0; j < n; ++j) {
            const int p = ipiv[j] - 1;
            if (p != j) {
                const double t = x[j];
                x[j] = x[p];
                x[p] = t;
            }
        }
        for (int k = 0; k < n; ++k)
            if (x[k] != 0.0)
                for (int i = k + 1; i < n; ++i) x[i] -= x[k] * A(i, k);
        for (int k = n - 1; k >= 0; --k)
            if (x[k] != 0.0) {
                x[k] /= A(k, k);
                for (int i = 0; i < k; ++i) x[i] -= x[k] * A(i, k);
            }
    }
}
