"""B200-native Bluebild imaging path (bipp drop-in): Gram matrix, generalized
eigensolver, energy levels, virtual visibilities, type-3 NUFFT and direct sum,
all on sm_100a through libbipp_b200.so."""
from .api import (  # noqa: F401
    BippError,
    Context,
    EigensolverError,
    GPUError,
    InMemoryDataset,
    InvalidParameterError,
    NufftSynthesis,
    NufftSynthesisOptions,
    Partition,
    Pipeline,
    communicator,
    config,
    default_context,
    domain_partition_grid,
    eigh,
    eigh_gram,
    eigh_gram_batched,
    eigh_gram_full,
    gram_matrix,
    image_synthesis,
    kernel_launch_count,
    nuft_sum,
    split_selection,
    virtual_vis,
)

__version__ = "0.1.0"
