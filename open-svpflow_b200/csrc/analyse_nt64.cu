// analyse_nt64.cu -- Analyse kernels with 64 threads per search direction, register budget
// cut for 4 resident CTAs per SM (see analyse_body.cuh).
#define SVPF_NT 64
#define SVPF_MINB 4
#define SVPF_VARIANT nt64
#include "analyse_body.cuh"
