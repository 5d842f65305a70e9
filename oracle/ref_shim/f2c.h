/* Test-infrastructure shim: the f2c scalar typedefs the reference's weight
   code (my_kriging_weights.h) declares its LAPACK arguments with. */
#ifndef ORACLE_SHIM_F2C_H
#define ORACLE_SHIM_F2C_H
typedef int integer;
typedef double doublereal;
#endif
