/*
 * ref_tbb20.cpp -- TEST INFRASTRUCTURE.  Compiles the reference's own
 * src/matchtbb.cu (included from where it lies, unmodified) with the round
 * cap lowered from NR_MAX_MATCH_ROUNDS (256) to NR_MATCH_ROUNDS + 1 (21), so
 * GraphMatchingTBB{Random,Weighted} run at most the 20 rounds of the GPU
 * fixed-round types 6 and 8 (matchgpu.cu:507-524, 705-722).  Rounds past the
 * point where every vertex is settled are no-ops in both, so the match[]
 * arrays agree; only the number of rand() values drawn differs (the GPU loop
 * always draws 20).
 */
#include "matchcpu.h"
#undef NR_MAX_MATCH_ROUNDS
#define NR_MAX_MATCH_ROUNDS (NR_MATCH_ROUNDS + 1)
#include "matchtbb.cu"
