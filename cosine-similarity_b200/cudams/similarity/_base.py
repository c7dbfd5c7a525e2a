"""Base class of the similarity plug-ins.

The reference subclasses matchms.similarity.BaseSimilarity.  matchms is a
third-party dependency; when it is installed the classes subclass it, so
matchms.calculate_scores accepts them and names their fields
<ClassName>_<field> (e.g. CudaCosineGreedy_score).  Without matchms a local
base with the same class attributes is used.
"""
try:  # pragma: no cover - depends on the environment
    from matchms.similarity.BaseSimilarity import BaseSimilarity  # type: ignore
except ImportError:  # matchms not installed
    import numpy as np

    class BaseSimilarity:  # type: ignore[no-redef]
        is_commutative = True
        score_datatype = np.float64

        def pair(self, reference, query):
            raise NotImplementedError

        def matrix(self, references, queries, array_type="numpy", is_symmetric=False):
            raise NotImplementedError

        def to_dict(self) -> dict:
            return {"__Similarity__": self.__class__.__name__,
                    **{k: v for k, v in self.__dict__.items() if not k.startswith("_")}}

__all__ = ["BaseSimilarity"]
