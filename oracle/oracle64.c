/* Binary64 twin of the oracle (TEST INFRASTRUCTURE ONLY, like oracle.c): the same
 * kernels evaluated in binary64, used to state the error of the binary32 step.
 * Exports te64_bind(double *D) and teor_<kernel>(uint32_t *M, const uint32_t *ARG),
 * where field values are read from and written to D (one double per memory word) and
 * parameter structs from M.  Build: oracle/Makefile (liboracle64.so). */
#define TE_ORACLE_F64 1
#include "oracle.c"
