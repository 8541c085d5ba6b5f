"""ibfs_b200 -- B200-native concurrent multi-source BFS (iBFS hot path).

The product is the C-ABI library ``libibfs.so`` (include/ibfs.h) with its
sm_100a kernels; this package is its Python binding and build helper.
"""
from .api import (  # noqa: F401
    LAYOUT_SOURCE_MAJOR,
    LAYOUT_VERTEX_MAJOR,
    MODE_AUTO,
    MODE_DEVICE_LOOP,
    MODE_PERSISTENT,
    MODE_PLAIN,
    Graph,
    GroupBy,
    IbfsError,
    Opts,
    Server,
    Stats,
    convert_text,
    csr_from_edges,
    default_opts,
    exported_names,
    gen_chung_lu,
    gen_grid,
    gen_rmat,
    graph_reader,
    groupby_csr,
    groupby_csr_maxhub,
    lib_path,
    read_csr,
    read_src_v,
    report,
    sample_sources,
    write_csr,
    write_src_v,
)
