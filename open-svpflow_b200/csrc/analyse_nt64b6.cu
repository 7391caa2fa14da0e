// analyse_nt64b6.cu -- Analyse kernels with 64 threads per search direction, register budget
// cut for 6 resident CTAs per SM (see analyse_body.cuh).
#define SVPF_NT 64
#define SVPF_MINB 6
#define SVPF_VARIANT nt64b6
#include "analyse_body.cuh"
