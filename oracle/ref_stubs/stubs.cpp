/* Bodies for the stand-in baseline reorderers: not on the SpMV path. */
#include <cstdlib>
void R_Cuthill_Mckee(int, int, int*, int*, unsigned int*) { std::abort(); }
void rabbit_order(int*, int*, int, int, unsigned int*) { std::abort(); }
