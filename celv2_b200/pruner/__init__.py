"""The learned partition / mode pruner (include/celv2_pruner.h).

``net``: the network's parameters and its training on the GPU through the library's own forward,
backward, loss and Adam kernels (torch tensors only hold the device memory); ``data``: training
records from the exhaustive engine on seeded synthetic clips; ``evaluate``: what pruning costs
(the chosen partitions' cost against the exhaustive search's) and saves; ``train``: the pipeline
that writes ``weights.npz``.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights.npz")


def load(path: str = WEIGHTS) -> dict:
    """The trained parameters and the thresholds chosen with them: {"params", "ref_threshold",
    "intra_threshold", "band"}."""
    import numpy as np

    z = np.load(path)
    return {"params": z["params"].astype(np.float32), "ref_threshold": float(z["ref_threshold"]),
            "intra_threshold": float(z["intra_threshold"]), "band": float(z["band"])}
