/* Stand-in for the PETSc headers, written for this project.
 *
 * Test infrastructure only. The reference's SVV.cpp includes <petsc.h>,
 * <petscvec.h> and <petscmat.h> but calls nothing from them; its Utils.h
 * names the Vec and Mat handle types in two declarations the oracle never
 * calls. These opaque handle types are all the compilation needs.
 */
#ifndef SE_ORACLE_PETSC_STUB_H
#define SE_ORACLE_PETSC_STUB_H
typedef struct se_stub_vec* Vec;
typedef struct se_stub_mat* Mat;
#endif
