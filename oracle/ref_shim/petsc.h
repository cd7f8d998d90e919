/* Shim for building the reference's pointwise kernels without PETSc.
 * Test infrastructure only: used by oracle/Makefile to compile the reference
 * fekernels into oracle/_ref/. PETSc's scalar types for a real, 32-bit-index,
 * double-precision build (the configuration PyLith uses). */
#pragma once
#include <math.h>
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscInt;
typedef int PetscErrorCode;
#define PETSC_SUCCESS 0
