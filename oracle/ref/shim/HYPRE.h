/* HYPRE IJ / ParCSR / PCG shim (test infrastructure for the oracle pin).
 * Serial CSR matrix and vectors; PCG restated from HYPRE 2.27.0's
 * hypre_PCGSolve with the identity preconditioner (the reference calls it
 * with BoomerAMG commented out, fluid_solver.h:1775-1787). */
#ifndef HS_SHIM_HYPRE_H
#define HS_SHIM_HYPRE_H
#include "mpi.h"
typedef int HYPRE_Int;
typedef double HYPRE_Complex;
typedef double HYPRE_Real;
typedef struct hs_ij_matrix *HYPRE_IJMatrix;
typedef struct hs_ij_matrix *HYPRE_ParCSRMatrix;
typedef struct hs_ij_vector *HYPRE_IJVector;
typedef struct hs_ij_vector *HYPRE_ParVector;
typedef struct hs_pcg *HYPRE_Solver;
typedef HYPRE_Int (*HYPRE_PtrToSolverFcn)(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
#define HYPRE_PARCSR 5555
HYPRE_Int HYPRE_Initialize(void);
HYPRE_Int HYPRE_Finalize(void);
HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm, HYPRE_Int, HYPRE_Int, HYPRE_Int, HYPRE_Int, HYPRE_IJMatrix *);
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int);
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix, HYPRE_Int, HYPRE_Int *, const HYPRE_Int *, const HYPRE_Int *, const HYPRE_Complex *);
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix, void **);
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm, HYPRE_Int, HYPRE_Int, HYPRE_IJVector *);
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int);
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector);
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector, HYPRE_Int, const HYPRE_Int *, const HYPRE_Complex *);
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector);
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector, void **);
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector, HYPRE_Int, const HYPRE_Int *, HYPRE_Complex *);
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector);
HYPRE_Int HYPRE_ParCSRPCGCreate(MPI_Comm, HYPRE_Solver *);
HYPRE_Int HYPRE_ParCSRPCGDestroy(HYPRE_Solver);
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_PCGSetMaxIter(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_PCGSetTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_PCGSetTwoNorm(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_PCGGetNumIterations(HYPRE_Solver, HYPRE_Int *);
HYPRE_Int HYPRE_PCGGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real *);
#endif
