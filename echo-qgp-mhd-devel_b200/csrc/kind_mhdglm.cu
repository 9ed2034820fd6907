// kind_mhdglm.cu -- kernels and launchers of one equation set (KIND_MHDGLM).
#include "launchers.cuh"

ECHO_INSTANTIATE(echo::KIND_MHDGLM)
