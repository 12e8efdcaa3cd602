/*
 * TEST INFRASTRUCTURE ONLY — the checker, never the product.
 *
 * Plain-C restatement of the reference (TNL) sparse hot path, used by tests/
 * and by the cpu_baseline leg of bench.py. Only tests/, __graft_entry__.smoke()
 * and bench.py may load it. The product (libb2sparse.so) never links it.
 *
 * Pinned against: (1) TNL's own unit-test golden values
 * (src/UnitTests/Matrices/SparseMatrixVectorProductTest.hpp) and (2) arrays and
 * results produced by TNL itself (oracle/_ref/libtnlref.so, built from the
 * reference headers), committed as fixtures under tests/golden/.
 */
#ifndef B2S_ORACLE_H
#define B2S_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b2so_matrix b2so_matrix;

/* format: 0 CSR (as given), 1 Ellpack, 2 SlicedEllpack(32), 3 ChunkedEllpack, 4 BiEllpack(32),
 *         5/6/7 SlicedEllpack with SliceSize 8/16/64
 * org:    0 ColumnMajorOrder (TNL Devices::Cuda default), 1 RowMajorOrder
 * real:   0 double, 1 float (values rounded to float, sums in float) */
b2so_matrix* b2so_create( int format, int org, int real, int rows, int cols,
                          const int* offsets, const int* columns, const double* values );
void b2so_destroy( b2so_matrix* m );

/* setRowCapacities( row_caps, or the per-row triplet counts when NULL ) +
 * setElement (add = 0) or addElement( .., 1 ) (add = 1) for every triplet in
 * order; NULL when a triplet lies outside the matrix or a row overflows. */
b2so_matrix* b2so_from_coo( int format, int org, int real, int rows, int cols, long long n, const int* ri,
                            const int* ci, const double* v, int add, const int* row_caps );
long long b2so_storage_size( const b2so_matrix* m );
void b2so_export_values( const b2so_matrix* m, double* out );
void b2so_export_columns( const b2so_matrix* m, int* out );
int b2so_meta_count( const b2so_matrix* m );
const char* b2so_meta_name( const b2so_matrix* m, int i );
long long b2so_meta_size( const b2so_matrix* m, int i );
void b2so_meta_get( const b2so_matrix* m, int i, long long* out );

/* y = alpha*A*x + beta*y over rows [begin, end); end == 0 means all rows. */
void b2so_spmv( const b2so_matrix* m, const double* x, double* y, double alpha, double beta, int begin, int end );

/* Matrices/MatrixPermutationApplier.h (rows: CSR only) and
 * SparseOperations_impl.h reorderSparseMatrix (CSR in, CSR out). */
int b2so_permute_rows( b2so_matrix* m, const int* perm );
int b2so_permute_columns( b2so_matrix* m, const int* iperm );
b2so_matrix* b2so_reorder( int rows, int cols, const int* offsets, const int* columns, const double* values,
                           const int* perm, const int* iperm );

/* ILU(0) of a CSR matrix (rows sorted, diagonal stored) and x = U^-1 L^-1 b;
 * fused bit 0 / 3: the factorization updates of a row's U / L part as fused
 * multiply-adds, bit 1 / 2: the forward / backward sums, bit 4: the sums in
 * groups of four rounded products, the remainder fused. -1 when a diagonal
 * entry is missing. */
int b2so_ilu0_apply( int real, int fused, int rows, const int* off, const int* col, const double* val, const double* b,
                     double* x );

/* SymmetricMatrix product: the CSR arrays hold the lower triangle (column <= row);
 * y = alpha A x + beta y over rows [begin, end) (end 0: all rows). */
void b2so_spmv_symmetric( int rows, const int* off, const int* col, const double* val, const double* x, double* y,
                          double alpha, double beta, int begin, int end );

/* Krylov solvers on a CSR matrix (TNL semantics). solver: 0 CG, 1 BiCGStab, 2 GMRES,
 * 3 TFQMR, 4 BiCGStab(ell). precond: 0 none, 1 Jacobi. gmres_variant: 0 CGS, 1 CGSR,
 * 2 MGS, 3 MGSR. ell: BiCGStab(ell)'s ell (0 = 1).
 * Returns 1 when converged (IterativeSolver::checkConvergence), 0 otherwise. */
int b2so_solve( int solver, int precond, int rows, const int* offsets, const int* columns, const double* values,
                const double* b, double* x, double rtol, long long maxit, int gmres_variant, int restart_min,
                int restart_max, int exact_residue, int ell, long long* iters, double* residue );

#ifdef __cplusplus
}
#endif
#endif
