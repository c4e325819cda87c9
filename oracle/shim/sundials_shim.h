/* Type-only stand-in for the SUNDIALS headers that the reference CAMP C
 * sources include when CAMP_USE_SUNDIALS is defined.  The reaction,
 * derivative and Jacobian code only needs these names to compile; nothing in
 * the oracle calls a SUNDIALS routine (the integrator is restated in
 * oracle/camp_oracle.c).  Test infrastructure only. */
#ifndef CAMP_ORACLE_SUNDIALS_SHIM_H
#define CAMP_ORACLE_SUNDIALS_SHIM_H
#define SUNDIALS_VERSION_MAJOR 3
typedef double realtype;
typedef int booleantype;
typedef long sunindextype;
typedef struct camp_oracle_nvector_opaque *N_Vector;
typedef struct camp_oracle_sunmatrix_opaque *SUNMatrix;
typedef struct camp_oracle_sunlinsol_opaque *SUNLinearSolver;
#define SUNTRUE 1
#define SUNFALSE 0
#endif
