"""topk_b200: exact top-k linear aggregation on B200 (sm_100a).

Drop-in for the TPAc path of avionicscode/TopK: the C ABI is include/topk_b200.h
(libtopk_b200.so, built by `python -m topk_b200.build`); this package is its
Python face, mirroring the reference's AA / TPAc algorithm-class API.
"""
from ._lib import (BATCH_AUTO, BATCH_BF16, BATCH_FP32, BATCH_LEARNED, BATCH_LOOP, DIST_ANTICORRELATED, DIST_CORRELATED,
                   DIST_INDEPENDENT, DIST_MIXED, MAX_D, MAX_K, MAX_Q, ORDER_MORTON, ORDER_PTA, ORDER_VTA,
                   ORDER_SLA, ORDER_VTA_THREADS, ORDER_KD, TopKError, load)
from .table import Table, binary_shape, csv_shape
from .tpac import AA, TA, TPAc, TPAr

__all__ = ["Table", "csv_shape", "binary_shape", "AA", "TA", "TPAc", "TPAr", "TopKError", "load", "MAX_K", "MAX_Q", "MAX_D", "DIST_CORRELATED",
           "DIST_INDEPENDENT", "DIST_ANTICORRELATED", "DIST_MIXED", "BATCH_AUTO", "BATCH_LOOP", "BATCH_FP32",
           "BATCH_BF16", "BATCH_LEARNED", "ORDER_MORTON", "ORDER_VTA", "ORDER_PTA",
           "ORDER_VTA_THREADS", "ORDER_SLA", "ORDER_KD"]
