// analyse_nt128p16.cu -- Analyse kernels for uint16 samples (the 10-bit extension), 128 threads
// per search direction, register budget cut for 2 resident CTAs per SM (see analyse_body.cuh).
#define SVPF_NT 128
#define SVPF_MINB 2
#define SVPF_VARIANT nt128p16
#define SVPF_PX16 1
#define SVPF_LOOKAHEAD 1
#include "analyse_body.cuh"
