"""B200-native exact brute-force Euclidean neighbour search.

A drop-in for the neighbour path of mlxlearn (``mlxlearn.neighbors``): the same
estimators, results contract and error behaviour, computed by a C-ABI CUDA
library for sm_100a (``libb200knn.so``, declared in ``include/b200knn.h``).
"""
__version__ = "0.1.0"
