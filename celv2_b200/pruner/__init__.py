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


THRESHOLDS = ("ref_threshold", "intra_threshold", "level_threshold", "mode_threshold", "band")


def load(path: str = WEIGHTS) -> dict:
    """The trained parameters and the thresholds chosen with them: {"params", "ref_threshold",
    "intra_threshold", "level_threshold", "mode_threshold", "band"}."""
    import numpy as np

    from .. import engine as E

    z = np.load(path)
    if z["params"].size != E.PRUNER_PARAMS or any(k not in z for k in THRESHOLDS):
        raise ValueError(f"{path} holds another network's weights (retrain: python -m celv2_b200.pruner.train)")
    out = {"params": z["params"].astype(np.float32)}
    for k in THRESHOLDS:
        out[k] = float(z[k])
    return out


def set_on(eng, wts: dict) -> None:
    """Turns the pruner on for engine `eng` with the weights and thresholds of `wts` (load())."""
    eng.set_pruner(wts["params"], *(wts[k] for k in THRESHOLDS))
