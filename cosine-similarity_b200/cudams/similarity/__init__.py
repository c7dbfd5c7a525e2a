from .CudaCosineGreedy import CudaCosineGreedy
from .CudaFingerprintSimilarity import CudaFingerprintSimilarity
from .CudaModifiedCosine import CudaModifiedCosine

__all__ = ["CudaCosineGreedy", "CudaFingerprintSimilarity", "CudaModifiedCosine"]
