// fk_mark_k6.cu -- marking-sieve variants of wheel family P0 = 6.
#define FK_MARK_P0 6
#include "fk_mark_k.cuh"
