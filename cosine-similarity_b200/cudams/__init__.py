"""cudams: pairwise mass-spectrum similarity on NVIDIA B200 (sm_100a).

Drop-in for the reference package of the same name: ``from cudams.similarity
import CudaCosineGreedy, CudaFingerprintSimilarity`` keeps working.  The
Python classes pack spectra on the host and call hand-written sm_100a CUDA
kernels in libcudams_b200.so through a ctypes C ABI (include/cudams_b200.h);
PyTorch is used only for device buffers and streams.  There is no CPU
fallback: without the native library or a B200 the calls raise.
"""
import warnings

from .__version__ import __version__

# Same warnings are given once (reference: cudams/__init__.py:18-19).
warnings.simplefilter("default", Warning)

__all__ = ["__version__"]
