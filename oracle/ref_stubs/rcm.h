/* Declaration-only stand-in for rcm/include/rcm.h (test infrastructure). */
#ifndef MR_REF_STUB_RCM_H
#define MR_REF_STUB_RCM_H
void R_Cuthill_Mckee(int n, int nz, int* rows, int* cols, unsigned int* permutation);
#endif
