/* Declaration-only stand-in for rabbitorder/include/rabbit_order.h; the real
 * library needs boost and libnuma, absent here (test infrastructure). */
#ifndef MR_REF_STUB_RABBIT_ORDER_H
#define MR_REF_STUB_RABBIT_ORDER_H
void rabbit_order(int* row_ind, int* col_ind, int nrow, int nnz, unsigned int* permutation);
#endif
