// fk_mark_k9.cu -- marking-sieve variants of wheel family P0 = 9.
#define FK_MARK_P0 9
#include "fk_mark_k.cuh"
