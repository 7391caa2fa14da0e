// analyse_nt128b3.cu -- Analyse kernels with 128 threads per search direction, register budget
// cut for 3 resident CTAs per SM (see analyse_body.cuh).
#define SVPF_NT 128
#define SVPF_MINB 3
#define SVPF_VARIANT nt128b3
#include "analyse_body.cuh"
