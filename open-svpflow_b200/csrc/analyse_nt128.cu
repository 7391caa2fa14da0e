// analyse_nt128.cu -- Analyse kernels with 128 threads per search direction, register budget
// cut for 2 resident CTAs per SM, with the level-0 look-ahead (see analyse_body.cuh).
#define SVPF_NT 128
#define SVPF_MINB 2
#define SVPF_VARIANT nt128
#define SVPF_LOOKAHEAD 1
#include "analyse_body.cuh"
