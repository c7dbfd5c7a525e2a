from .CudaCosineGreedy import CudaCosineGreedy
from .CudaFingerprintSimilarity import CudaFingerprintSimilarity

__all__ = ["CudaCosineGreedy", "CudaFingerprintSimilarity"]
