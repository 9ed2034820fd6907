// kind_hd.cu -- kernels and launchers of one equation set (KIND_HD).
#include "launchers.cuh"

ECHO_INSTANTIATE(echo::KIND_HD)
