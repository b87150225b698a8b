"""B200-native implementation of BootCMatchGX's single-rank FCG + BCMG (matching-based
aggregation AMG) solver path. All computation runs in libbcmgx.so (hand-written sm_100a
kernels behind the C ABI of include/bcmgx.h); this package is the host-side binding."""
from ._lib import BcmgxError, LIB_PATH, lib  # noqa: F401
from .api import (  # noqa: F401
    Batch, Dist, Hierarchy, diffusion_7p, edge_weights, init_from_file, init_from_properties_file, laplacian,
    laplacian_3d, laplacian_3d_size, params_default, params_to_dict, prec_finalize, prec_setup,
    nccl_comm, nccl_comm_destroy, nccl_unique_id, read_laplacian_cfg, read_matrix_market, set_params, solve,
    spmm, spmv, suitor_matching,
)

__all__ = [
    "Batch", "BcmgxError", "Dist", "Hierarchy", "diffusion_7p", "edge_weights", "init_from_file",
    "init_from_properties_file", "laplacian", "laplacian_3d", "laplacian_3d_size", "lib",
    "nccl_comm", "nccl_comm_destroy", "nccl_unique_id",
    "params_default", "params_to_dict", "prec_finalize", "prec_setup", "read_laplacian_cfg",
    "read_matrix_market", "set_params", "solve", "spmm", "spmv", "suitor_matching",
]
