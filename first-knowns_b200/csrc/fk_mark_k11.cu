// fk_mark_k11.cu -- marking-sieve variants of wheel family P0 = 11.
#define FK_MARK_P0 11
#include "fk_mark_k.cuh"
