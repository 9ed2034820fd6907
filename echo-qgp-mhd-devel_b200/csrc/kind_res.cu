// kind_res.cu -- kernels and launchers of one equation set (KIND_RES,
// resistive MHD; single grid only: the batched mode rejects MHD = 2).
#include "launchers.cuh"

ECHO_INSTANTIATE_GRID(echo::KIND_RES)
