// fk_mark_k7.cu -- marking-sieve variants of wheel family P0 = 7.
#define FK_MARK_P0 7
#include "fk_mark_k.cuh"
