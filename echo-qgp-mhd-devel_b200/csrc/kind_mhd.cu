// kind_mhd.cu -- kernels and launchers of one equation set (KIND_MHD).
#include "launchers.cuh"

ECHO_INSTANTIATE(echo::KIND_MHD)
