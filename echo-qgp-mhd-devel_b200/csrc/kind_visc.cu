// kind_visc.cu -- kernels and launchers of one equation set (KIND_VISC).
#include "launchers.cuh"

ECHO_INSTANTIATE(echo::KIND_VISC)
