from .CudaCosineGreedy import CudaCosineGreedy
from .CudaFingerprintSimilarity import CudaFingerprintSimilarity
from .CudaIntersectMz import CudaIntersectMz
from .CudaModifiedCosine import CudaModifiedCosine
from .CudaPrecursorMzMatch import CudaParentMassMatch, CudaPrecursorMzMatch

__all__ = ["CudaCosineGreedy", "CudaFingerprintSimilarity", "CudaIntersectMz",
           "CudaModifiedCosine", "CudaParentMassMatch", "CudaPrecursorMzMatch"]
