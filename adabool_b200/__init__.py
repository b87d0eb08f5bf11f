"""adabool_b200 -- B200-native Boolean filtering over compressed inverted lists.

Host-side mirror of the reference's operator interface (yxr620/AdaBool):

    ivf_list::BuildFrom (src/AdaBool/inverted_list.h:348)   -> Index.BuildFrom / Index.from_coo
    ivf_list::Prepare(keys) (inverted_list.h:481)           -> Index.Prepare(keys)
    ivf_list::Prepare(len, bitmap) (inverted_list.h:530)    -> Index.Prepare(len, bitmap)
    ivf_list::PrepareBatch / PrepareBatchDevice (:564,:591) -> Index.PrepareBatch / PrepareBatchDevice
    ListUnion_dense / ListUnion_sparse (test/adsfilter_q_all.cu:26,64)
    BatchListUnion_dense / BatchListUnion_sparse (test/adsfilter_batch.cu:28,39)
    CollectIdsFromBitmap (test/adsfilter_batch.cu:82)       -> CollectIdsFromBitmap (device compaction)

Every call goes through libadabool.so; device buffers are torch CUDA tensors.
"""
from ._native import (AbfError, PATH_AUTO, PATH_HYBRID, PATH_NAMES, PATH_PROBE, PATH_TILE, PATH_UNION,
                      lib)
from .index import (Index, Worker, Workspace, ListUnion_dense, ListUnion_sparse, BatchListUnion_dense,
                    BatchListUnion_sparse, BatchCollectIds, CollectIdsFromBitmap, launch_count)

__all__ = ["AbfError", "Index", "Worker", "Workspace", "ListUnion_dense", "ListUnion_sparse",
           "BatchListUnion_dense", "BatchListUnion_sparse", "BatchCollectIds", "CollectIdsFromBitmap", "launch_count", "lib",
           "PATH_AUTO", "PATH_PROBE", "PATH_UNION", "PATH_HYBRID", "PATH_TILE", "PATH_NAMES"]
