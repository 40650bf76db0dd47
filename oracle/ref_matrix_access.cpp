/*
 * Test infrastructure only (oracle build).
 *
 * Read access to the reference's fun3d::Matrix (matrix/matrix.h:7-93) so tests
 * can compare the BSR Jacobian of src/fill.c and the ILU(0) factor of
 * matrix/ilu.cpp:49-138 block by block.  This file is compiled with
 * -Dprivate=public; the reference's header is included unchanged.
 */
#include <stddef.h>
#include "matrix.h"

extern "C" {

size_t ref_matrix_rows(void *ptr)
{
  return ((fun3d::Matrix *) ptr)->nrows;
}

/* BSR of A: row pointers (nrows+1), sorted columns, diagonal positions and
   4x4 row-major blocks. */
void ref_matrix_bsr(void *ptr, const unsigned int **ia, const unsigned int **ja,
                    const unsigned int **d, const double **a)
{
  fun3d::Matrix *m = (fun3d::Matrix *) ptr;
  *ia = m->A->i;
  *ja = m->A->j;
  *d = m->A->d;
  *a = m->A->a;
}

/* Number of forward (TL) and backward (TU) levels of matrix/init.cpp:194-274. */
void ref_matrix_levels(void *ptr, unsigned int *nl, unsigned int *nu)
{
  fun3d::Matrix *m = (fun3d::Matrix *) ptr;
  *nl = m->TL->n;
  *nu = m->TU->n;
}

}
