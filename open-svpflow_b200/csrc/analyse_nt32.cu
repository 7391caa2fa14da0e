// analyse_nt32.cu -- Analyse kernels with 32 threads per search direction, register budget
// cut for 8 resident CTAs per SM (see analyse_body.cuh).
#define SVPF_NT 32
#define SVPF_MINB 8
#define SVPF_VARIANT nt32
#include "analyse_body.cuh"
